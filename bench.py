"""Benchmark of the fused VISCOPLASTIC-LBM time step on B200.

Workload (one "step" = one fused time step over the whole lattice): the
regularized Bingham plane channel, D3Q19, 256 x 128 x 64, plastic tau 0.8
(eta_p = 0.1), yield stress 1e-5, body force gx = 5e-6, bounce-back walls at
y = 0 and y = NY-1, periodic x and z, rho = 1 u = 0 initial state, FP32
populations (the BASELINE second configuration).  Synthetic by construction:
the lattice state evolves from the equilibrium initial condition.

Metric: MLUPS (million lattice-node updates per second, all nodes counted as
the reference does, src/CUDA/main.cu:411), plus the HBM-roofline fraction of
the fused kernel.  Multi-GPU runs are independent replicas (the path is one
lattice per GPU); value = all ranks' node updates / max-over-ranks time.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

`--vel-set 27` and `--size NX NY NZ` run the same channel on another velocity
set or lattice (the workload name says which); they exist for profiling runs.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "viscoplastic-lbm_b200"))

NX, NY, NZ, Q = 256, 128, 64, 19
WORKLOAD = "d3q19_regularized_bingham_channel_256x128x64"
METRIC = "MLUPS"
L2_BYTES = 126 * 2 ** 20


def set_workload(q, nx, ny, nz):
    global NX, NY, NZ, Q, WORKLOAD
    NX, NY, NZ, Q = nx, ny, nz, q
    WORKLOAD = f"d3q{q}_regularized_bingham_channel_{nx}x{ny}x{nz}"


def config_dict(storage="f32"):
    pop_mb = Q * NX * NY * NZ * {"f16": 2, "bf16": 2, "f64": 8}.get(storage, 4) / 1e6
    rel = "larger" if pop_mb * 1e6 > L2_BYTES else "smaller"
    return {"workload": WORKLOAD, "nx": NX, "ny": NY, "nz": NZ, "velocity_set": f"D3Q{Q}",
            "collision": "regularized", "rheology": "bingham", "tau_p": 0.8, "yield_stress": 1e-5,
            "gx": 5e-6, "walls": "y (half-way bounce-back)", "periodic": "x,z", "storage": storage,
            "streaming": "AA in-place",
            "l2_policy": f"population array ({pop_mb:.0f} MB) {rel} than the 126 MB L2",
            "parallelism": "replicas"}


def make_cfg(vlbm, storage=0):
    return vlbm.Config.default(nx=NX, ny=NY, nz=NZ, vel_set=Q, collision=vlbm.OP_REGULARIZED,
                               rheology=vlbm.BINGHAM, eta_p=(0.8 - 0.5) / 3.0, yield_stress=1e-5,
                               fx=5e-6, storage=storage)


def measured_peak():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


TRAFFIC_PROFILES = {
    # (storage, resolved layout) -> ncu summary of that kernel on this workload
    ("f32", "natural"): "fused_step_d3q19_bingham_256x128x64.md",
    ("f32", "zpair"): "fused_step2_d3q19_bingham_f32_256x128x64.md",
    ("f16", "zpair"): "fused_step2_d3q19_bingham_f16_256x128x64.md",
}


def committed_traffic(storage, layout):
    """dram read+write bytes per launch of the fused kernel from the committed ncu summary
    of the same storage and layout (None when no capture of that kernel is committed)."""
    if (Q, NX, NY, NZ) != (19, 256, 128, 64):
        return None            # captures are committed for the default workload only
    if layout == "auto":   # the library's AUTO rule for D3Q19 with an even nz
        layout = "natural" if storage == "f32" else "zpair"
    name = TRAFFIC_PROFILES.get((storage, layout))
    if name is None:
        return None
    try:
        for line in open(os.path.join(REPO, "profiles", name)):
            if line.startswith("traffic_bytes_per_launch:"):
                return float(line.split(":", 1)[1].strip())
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.out = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)

    def start(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.out, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.out.flush()
        rows = []
        for line in open(self.out.name):
            p = [x.strip() for x in line.split(",")]
            if len(p) >= 9:
                rows.append(p)
        os.unlink(self.out.name)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = max((float(r[2]) for r in rows if r[2].replace(".", "").isdigit()), default=None)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": reasons,
                "samples": len(rows)}


def load_oracle():
    """The FP64 oracle module, oracle/oracle.py, loaded by its path (the
    repository's oracle/ folder would otherwise import as an empty namespace
    package when the repository root is on sys.path)."""
    import importlib.util
    name = "vlbm_bench_oracle"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, os.path.join(REPO, "oracle", "oracle.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def oracle_cfg(oracle):
    """The workload's configuration for the oracle (oracle.Config: vlbm_config's
    layout filled without loading libvlbm)."""
    return oracle.Config.default(nx=NX, ny=NY, nz=NZ, vel_set=Q, collision=0, rheology=1,
                                 eta_p=(0.8 - 0.5) / 3.0, yield_stress=1e-5, fx=5e-6)


def cpu_baseline(seconds_budget=15.0, max_steps=None):
    """The FP64 OpenMP oracle (restated reference step) on the host cores, on the
    full workload lattice for as many steps as fit in the time budget.  Loads
    only oracle/liboracle.so: the node map is the oracle's own restatement of
    the reference builder."""
    oracle = load_oracle()
    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    o = oracle.Oracle(oracle_cfg(oracle), oracle.plates_y_map(NX, NY, NZ))
    o.step(1)
    steps, t0 = 0, time.perf_counter()
    while time.perf_counter() - t0 < seconds_budget and (max_steps is None or steps < max_steps):
        o.step(1)
        steps += 1
    dt = time.perf_counter() - t0
    o.close()
    mlups = steps * NX * NY * NZ / dt / 1e6
    return {"value": mlups, "unit": METRIC, "cores": threads, "kind": "port",
            "sample": f"full {NX}x{NY}x{NZ} workload lattice, {steps} steps after 1 untimed, FP64 oracle, "
                      f"{dt:.1f} s"}


def cube_leg(vlbm, torch, device, steps=200, warmup=10, n=256):
    """Regularized Bingham channel at n^3 for D3Q19 and D3Q27 with FP32 and FP16
    storage (AUTO layout, autotuned launch): MLUPS, algorithmic GB/s and the
    fraction of the measured copy bandwidth, timed with CUDA events over
    `steps` steps (the population arrays, 0.6-1.8 GB, exceed the 126 MB L2)."""
    peak, _ = measured_peak()
    out = {"lattice": f"{n}x{n}x{n}", "steps": steps,
           "case": "regularized Bingham, tau_p 0.8, yield 1e-5, gx 5e-6, walls y, periodic x,z"}
    for q in (19, 27):
        for name, st in (("f32", vlbm.STORE_F32), ("f16", vlbm.STORE_F16)):
            cfg = vlbm.Config.default(nx=n, ny=n, nz=n, vel_set=q, collision=vlbm.OP_REGULARIZED,
                                      rheology=vlbm.BINGHAM, eta_p=0.1, yield_stress=1e-5, fx=5e-6, storage=st)
            cfg.device = device
            sim = vlbm.Simulation(cfg, builder=vlbm.BUILDER_PLATES_Y)
            stream = torch.cuda.Stream()
            sim.set_stream(stream.cuda_stream)
            sim.autotune()
            sim.init_equilibrium(1.0, 0, 0, 0)
            sim.step(warmup)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            sim.step(steps)
            e1.record(stream)
            torch.cuda.synchronize()
            sim.sync()
            ms = e0.elapsed_time(e1)
            nodes = n ** 3
            bpn = sim.info().bytes_per_node_step
            mlups = nodes * steps / (ms / 1e3) / 1e6
            gbs = bpn * mlups * 1e6 / 1e9
            out[f"d3q{q}_{name}"] = {"mlups": mlups, "achieved_gbs": gbs, "frac": gbs / peak,
                                     "bytes_per_node": bpn, "variant": sim.info().last_kernel_variant,
                                     "layout": ("natural", "zpair", "zpair_blocked")[sim.info().layout]}
            sim.close()
        out[f"d3q{q}_f16_over_f32"] = out[f"d3q{q}_f16"]["mlups"] / out[f"d3q{q}_f32"]["mlups"]
    return out


def cavity_leg(vlbm, torch, device, steps=200, warmup=10, n=256):
    """The Power-Law lid-driven cavity: D3Q27 regularized, closed box of n^3
    nodes (all six faces half-way bounce-back, the lid y = NY-1 moving at
    u = 0.05 in x), flow index 0.5 / 1.0 / 1.5 with the consistency that makes
    Re = U^(2-n) L^n / K = 400 (L = n nodes), FP32 / FP16 / BF16 deviation
    storage, AUTO layout and an autotuned launch.  MLUPS and the fraction of the
    measured copy bandwidth for the 2*Q*s population bytes (the Power-Law
    viscosity state adds 8 B per node, reported beside them)."""
    peak, _ = measured_peak()
    out = {"lattice": f"{n}x{n}x{n}", "steps": steps, "velocity_set": "D3Q27", "re": 400, "lid_u": 0.05}
    for n_index in (0.5, 1.0, 1.5):
        k = 0.05 ** (2.0 - n_index) * n ** n_index / 400.0
        for name, st in (("f32", vlbm.STORE_F32), ("f16", vlbm.STORE_F16), ("bf16", vlbm.STORE_BF16)):
            cfg = vlbm.Config.default(nx=n, ny=n, nz=n, vel_set=27, collision=vlbm.OP_REGULARIZED,
                                      rheology=vlbm.POWERLAW, n_index=n_index, k_consistency=k, gamma0=0.0,
                                      ux_bc=[0, 0.05], storage=st)
            cfg.device = device
            sim = vlbm.Simulation(cfg, builder=vlbm.BUILDER_LID_CAVITY_CLOSED)
            stream = torch.cuda.Stream()
            sim.set_stream(stream.cuda_stream)
            variant = sim.autotune()
            sim.init_equilibrium(1.0, 0, 0, 0)
            sim.step(warmup)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            sim.step(steps)
            e1.record(stream)
            torch.cuda.synchronize()
            sim.sync()
            ms = e0.elapsed_time(e1)
            bpn = sim.info().bytes_per_node_step
            mlups = n ** 3 * steps / (ms / 1e3) / 1e6
            gbs = bpn * mlups * 1e6 / 1e9
            out[f"n{n_index}_{name}"] = {"mlups": mlups, "achieved_gbs": gbs, "frac": gbs / peak,
                                         "bytes_per_node": bpn, "state_bytes_per_node": 8, "k_consistency": k,
                                         "variant": variant}
            sim.close()
    return out


def sphere_pack(n, radius, box, gap=1.0, seed=42):
    """Non-overlapping sphere centres by rejection sampling: at least `gap`
    lattice units between spheres and to the walls (numpy default_rng(seed))."""
    import numpy as np
    rng = np.random.default_rng(seed)
    lo = radius + gap
    out = []
    while len(out) < n:
        c = lo + rng.random(3) * (np.array(box, dtype=float) - 1 - 2 * lo)
        if all(np.linalg.norm(c - o) >= 2 * radius + gap for o in out):
            out.append(c)
    return out


def ibm_leg(vlbm, torch, device, steps=50, warmup=5):
    """The IBM configuration: 192x192x384 closed box, D3Q19 regularized Bingham
    (tau_p 0.8, yield 1e-5), gravity -z, 64 movable spheres of radius 8
    (density ratio 1.5, non-overlapping, default_rng(42)), 3 direct-forcing
    iterations, Hertz-Mindlin contacts (E 1e5, Poisson 0.3, friction 0.3).
    Timed with and without the spheres on the same lattice."""
    import numpy as np
    nx, ny, nz = 192, 192, 384
    cfg = vlbm.Config.default(nx=nx, ny=ny, nz=nz, vel_set=19, collision=vlbm.OP_REGULARIZED,
                              rheology=vlbm.BINGHAM, eta_p=0.1, yield_stress=1e-5)
    cfg.device = device
    ibm = vlbm.IbmConfig.default(max_iterations=3, gx=0.0, gy=0.0, gz=-1e-5, wall_x=1, wall_y=1, wall_z=1,
                                 particle_young=1e5, wall_young=1e5, particle_poisson=0.3, wall_poisson=0.3,
                                 pp_friction=0.3, pw_friction=0.3)
    centres = sphere_pack(64, 8.0, (nx, ny, nz))
    spheres = [vlbm.Sphere(diameter=16.0, cx=float(c[0]), cy=float(c[1]), cz=float(c[2]), density=1.5, movable=1)
               for c in centres]
    out = {"lattice": f"{nx}x{ny}x{nz}", "spheres": 64, "radius": 8, "mdf_iterations": 3, "steps": steps}
    for with_spheres in (False, True):
        sim = vlbm.Simulation(cfg, builder=vlbm.BUILDER_CLOSED_BOX)
        stream = torch.cuda.Stream()
        sim.set_stream(stream.cuda_stream)
        sim.autotune()
        if with_spheres:
            sim.add_spheres(ibm, spheres)
        sim.step(warmup)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        sim.step(steps)
        e1.record(stream)
        torch.cuda.synchronize()
        sim.sync()
        ms = e0.elapsed_time(e1) / steps
        key = "with_spheres" if with_spheres else "fluid_only"
        out[key] = {"ms_per_step": ms, "mlups": nx * ny * nz / (ms / 1e3) / 1e6}
        if with_spheres:
            info = sim.info()
            out["lagrangian_nodes"] = info.n_lagrangian_nodes
            z = np.array([p.pos[2] for p in sim.particles(64)])
            out["mean_sphere_z_drop"] = float(np.mean([c[2] for c in centres]) - z.mean())
        sim.close()
    out["ibm_ms_per_step"] = out["with_spheres"]["ms_per_step"] - out["fluid_only"]["ms_per_step"]
    return out


def serving_requests(vlbm, n, step_scale, seed=2024):
    """A seeded sample of the Bingham-duct serving stream.

    Per request: nx uniform in [32, 256], ny = nz uniform in [16, 96], D3Q19 or
    D3Q27 at 50/50, tau_p uniform in [0.6, 1.2], Bingham number log-uniform in
    [0.1, 10], 2,000-20,000 steps (times step_scale), 20 % carrying 1-4
    movable spheres of radius 4-6 lattice units, FP16-deviation storage.  The
    duct has walls in y and z and is periodic in x; the body force gives a
    plane-Poiseuille centre-line speed of 0.02 across the duct width, and the
    yield stress follows from the Bingham number with that speed and width.
    """
    import numpy as np
    rng = np.random.default_rng(seed)
    out = []
    for tag in range(n):
        nx = int(rng.integers(32, 257))
        ny = int(rng.integers(16, 97))
        q = 19 if rng.random() < 0.5 else 27
        tau = float(rng.uniform(0.6, 1.2))
        nu = (tau - 0.5) / 3.0
        bn = float(10 ** rng.uniform(-1, 1))
        u, h = 0.02, ny - 2
        cfg = vlbm.Config.default(nx=nx, ny=ny, nz=ny, vel_set=q, collision=vlbm.OP_REGULARIZED,
                                  rheology=vlbm.BINGHAM, eta_p=nu, yield_stress=bn * nu * u / h,
                                  fx=8.0 * nu * u / (h * h), storage=vlbm.STORE_F16)
        steps = max(1, int(round(int(rng.integers(2000, 20001)) * step_scale)))
        spheres = []
        if rng.random() < 0.2:
            for _ in range(int(rng.integers(1, 5))):
                r = float(rng.uniform(4, 6))
                if ny - 2 * r - 5 <= 0:   # the duct is too narrow for this sphere
                    continue
                for _try in range(50):
                    c = (float(rng.uniform(0, nx)), float(rng.uniform(r + 2, ny - r - 3)),
                         float(rng.uniform(r + 2, ny - r - 3)))
                    if all((c[0] - o.cx) ** 2 + (c[1] - o.cy) ** 2 + (c[2] - o.cz) ** 2 > (r + o.diameter / 2 + 1) ** 2
                           for o in spheres):
                        spheres.append(vlbm.Sphere(diameter=2 * r, cx=c[0], cy=c[1], cz=c[2], density=1.5, movable=1))
                        break
        out.append(dict(tag=tag, cfg=cfg, steps=steps, spheres=spheres, nodes=nx * ny * ny))
    return out


SERVING_IBM = dict(max_iterations=1, gx=0.0, gy=0.0, gz=-1e-5, wall_x=0, wall_y=1, wall_z=1)


def serving_leg(vlbm, n_req=512, step_scale=0.25, rate=20.0, budget_gb=64.0, max_resident=64, seed=2024,
                plain_repeats=1):
    """Continuous batching against plain one-at-a-time solves on one arrival stream.

    Both arms see the same Poisson arrivals (rate requests/s).  The plain arm
    serves the requests first-in first-out with one simulation at a time
    through the public API (create, node map, spheres, step, read ux,
    destroy), each in its own best layout (LAYOUT_AUTO: z-paired FP16 where NZ
    is even); it runs `plain_repeats` times and the fastest run is compared.
    The batched arm submits each request to a vlbm_server when it arrives (the
    server runs every lattice in the natural layout), pumps it and fetches each
    result when it completes (the server keeps the last 256 results).  Where
    the two arms' layouts differ they round half-precision stores with
    different random streams, so their ux fields are compared by relative L2.
    Latency = time the result is handed back - arrival time; solves/s =
    requests / (last completion - first arrival).
    """
    import numpy as np
    reqs = serving_requests(vlbm, n_req, step_scale, seed)
    arrivals = np.cumsum(np.random.default_rng(seed + 1).exponential(1.0 / rate, n_req))
    arrivals -= arrivals[0]
    ibm = vlbm.IbmConfig.default(**SERVING_IBM)
    lu = float(sum(r["nodes"] * r["steps"] for r in reqs))

    def plain_run():
        t0 = time.perf_counter()
        lat, ux = [], {}
        for r, a in zip(reqs, arrivals):
            now = time.perf_counter() - t0
            if now < a:
                time.sleep(a - now)
            sim = vlbm.Simulation(r["cfg"], builder=vlbm.BUILDER_DUCT_YZ)
            if r["spheres"]:
                sim.add_spheres(ibm, r["spheres"])
            sim.step(r["steps"])
            sim.sync()
            ux[r["tag"]] = sim.macroscopics()["ux"].ravel().copy()
            sim.close()
            lat.append(time.perf_counter() - t0 - a)
        return time.perf_counter() - t0, lat, ux

    plain_runs = [plain_run() for _ in range(max(1, plain_repeats))]
    plain_span, plain_lat, plain_ux = min(plain_runs, key=lambda t: t[0])
    plain_spans = [t[0] for t in plain_runs]

    srv = vlbm.Server(device=0, hbm_budget_bytes=int(budget_gb * 2 ** 30), max_resident=max_resident)
    t0 = time.perf_counter()
    nxt, done, arrive_at, got_ux = 0, [], {}, {}
    nodes = {r["tag"]: r["nodes"] for r in reqs}
    while len(done) < n_req:
        now = time.perf_counter() - t0
        while nxt < n_req and arrivals[nxt] <= now:
            r = reqs[nxt]
            srv.submit(r["cfg"], vlbm.BUILDER_DUCT_YZ, r["steps"], r["tag"], r["spheres"], ibm)   # server: natural
            arrive_at[r["tag"]] = arrivals[nxt]
            nxt += 1
        st = srv.stats()
        if st["resident"] == 0 and st["queued"] == 0:
            time.sleep(max(0.0, arrivals[nxt] - (time.perf_counter() - t0)))
            continue
        for c in srv.pump(200):
            if c.status != vlbm.OK:
                raise RuntimeError(f"serving request {c.tag} failed with status {c.status}")
            got_ux[c.tag] = srv.fetch(c.tag, nodes[c.tag])
            done.append((c, time.perf_counter() - t0))
    batched_span = time.perf_counter() - t0
    host_profile = srv.profile()
    rels = []
    for c, _ in done:
        ref, got = plain_ux[c.tag], got_ux[c.tag]
        rels.append(float(np.linalg.norm(got - ref) / max(1e-30, np.linalg.norm(ref))))
    srv.close()
    batched_lat = [t_ret - arrive_at[c.tag] for c, t_ret in done]

    def arm(span, lat):
        return {"solves_per_s": n_req / span, "p50_s": float(np.percentile(lat, 50)),
                "p99_s": float(np.percentile(lat, 99)), "mlups": lu / span / 1e6, "makespan_s": span}

    batched, plain = arm(batched_span, batched_lat), arm(plain_span, plain_lat)
    plain["solves_per_s_runs"] = [n_req / t for t in plain_spans]
    return {"requests": n_req, "step_scale": step_scale, "arrival_rate_per_s": rate, "seed": seed,
            "with_spheres": sum(1 for r in reqs if r["spheres"]), "lattice_updates": lu,
            "batched": batched, "plain": plain, "speedup_solves": batched["solves_per_s"] / plain["solves_per_s"],
            "server_host_seconds": host_profile, "ux_rel_l2_vs_plain": {"median": float(np.median(rels)),
                                                                        "max": float(np.max(rels))},
            "sample": f"{n_req} requests of the Bingham-duct serving stream, step counts x{step_scale}"}


def shard_leg(args, rank, world, local):
    """The channel split into z-slabs, one per rank (zslab.ZSlab): NX x NY x
    (NZ x world) nodes, NZ planes per GPU, halos traded over NCCL around every
    odd step (a single rank trades with itself).  One JSON line, weak scaling."""
    import torch
    import vlbm
    import zslab
    dist = None
    if world > 1:
        import torch.distributed as dist
    storage = {"f32": vlbm.STORE_F32, "f16": vlbm.STORE_F16, "bf16": vlbm.STORE_BF16}[args.storage]
    cfg = make_cfg(vlbm, storage)
    cfg.nz = NZ * world
    cfg.layout = {"auto": vlbm.LAYOUT_AUTO, "natural": vlbm.LAYOUT_NATURAL, "zpair": vlbm.LAYOUT_ZPAIR}[args.layout]
    cfg.device = local
    slab = zslab.ZSlab(cfg, vlbm.BUILDER_PLATES_Y, autotune=True)
    stream = slab.stream
    slab.sim.init_equilibrium(1.0, 0, 0, 0)
    slab.step(args.warmup)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    slab.step(args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    clk = clocks.stop()
    slab.sim.sync()
    t = torch.tensor([ms], device="cuda")
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.barrier()
    ms_max = float(t.item())
    n_own = NX * NY * slab.n
    value = NX * NY * cfg.nz * args.steps / (ms_max / 1e3) / 1e6
    info = slab.sim.info()
    odd_steps = args.steps // 2
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": args.storage, "data": "synthetic",
        "config": dict(config_dict(args.storage), workload="D3Q%d channel %dx%dx%d split into %d z-slabs of %d planes"
                       % (Q, NX, NY, cfg.nz, world, slab.n), parallelism="z-slab x%d" % world),
        "layout": ("natural", "zpair", "zpair_blocked")[info.layout],
        "halo_bytes_per_message": slab.sim.halo_bytes(),
        "halo_messages_per_odd_step": 4,
        "own_nodes_per_gpu": n_own,
        "gpu_launches": args.steps * (1 if info.layout == 0 else 2) + odd_steps * 4,
        "clocks": clk,
    }
    slab.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()
    return 0


def run_reference(args, rank, world):
    """The reference arm: the FP64 OpenMP oracle, the reference's step restated
    on the host cores (the reference itself has no CPU path), on the full
    workload lattice.  Rank 0 alone runs it; the other ranks exit without work.
    It imports neither libvlbm nor torch."""
    if rank != 0:
        return 0
    budget = float(os.environ.get("VLBM_REFERENCE_BUDGET_S", "120"))
    base = cpu_baseline(seconds_budget=budget, max_steps=args.steps)
    line = {"impl": "reference", "metric": METRIC, "value": base["value"], "unit": METRIC,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": config_dict("f32"), "cpu_baseline": base,
            "e2e": {"value": base["value"], "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="vlbm", choices=["vlbm", "reference"])
    ap.add_argument("--storage", default="f32", choices=["f32", "f16", "bf16"])
    ap.add_argument("--layout", default="auto", choices=["auto", "natural", "zpair"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--no-cube", action="store_true", help="skip the 256^3 D3Q19/D3Q27 FP32/FP16 leg")
    ap.add_argument("--no-ibm", action="store_true", help="skip the 64-sphere IBM leg")
    ap.add_argument("--no-cavity", action="store_true", help="skip the 256^3 Power-Law lid-cavity leg")
    ap.add_argument("--ibm-steps", type=int, default=50, help="timed steps of the 64-sphere IBM leg")
    ap.add_argument("--vel-set", type=int, default=19, choices=[19, 27])
    ap.add_argument("--shard", action="store_true",
                    help="one lattice split into z-slabs over the ranks (NZ planes per GPU) instead of replicas")
    ap.add_argument("--size", type=int, nargs=3, default=[256, 128, 64], metavar=("NX", "NY", "NZ"))
    ap.add_argument("--e2e-steps", type=int, default=3000,
                    help="steps of the end-to-end leg (its host copies are amortised over them)")
    ap.add_argument("--serving-requests", type=int, default=512)
    ap.add_argument("--serving-plain-repeats", type=int, default=1,
                    help="runs of the plain one-at-a-time arm; the fastest is compared")
    ap.add_argument("--serving-step-scale", type=float, default=0.25)
    ap.add_argument("--serving-rate", type=float, default=200.0)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    set_workload(args.vel_set, *args.size)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        return run_reference(args, rank, world)

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    if args.shard:
        return shard_leg(args, rank, world, local)
    import vlbm

    storage = {"f32": vlbm.STORE_F32, "f16": vlbm.STORE_F16, "bf16": vlbm.STORE_BF16}[args.storage]
    cfg = make_cfg(vlbm, storage)
    cfg.layout = {"auto": vlbm.LAYOUT_AUTO, "natural": vlbm.LAYOUT_NATURAL, "zpair": vlbm.LAYOUT_ZPAIR}[args.layout]
    cfg.device = local
    sim = vlbm.Simulation(cfg, builder=vlbm.BUILDER_PLATES_Y)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    sim.set_stream(stream.cuda_stream)
    variant = sim.autotune()
    sim.init_equilibrium(1.0, 0, 0, 0)

    sim.step(args.warmup)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    sim.step(args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    clk = clocks.stop()
    sim.sync()
    t = torch.tensor([ms], device="cuda")
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.barrier()
    ms_max = float(t.item())
    N = NX * NY * NZ
    value = world * N * args.steps / (ms_max / 1e3) / 1e6

    info = sim.info()
    bytes_per_node = info.bytes_per_node_step
    achieved_gbs = bytes_per_node * N / (ms / 1e3 / args.steps) / 1e9
    peak, peak_kind = measured_peak()
    # the layout the autotuner kept (one launch per step in the natural layout;
    # the pair step adds the launch over the tiles that hold the channel's walls)
    chosen_layout = ("natural", "zpair", "zpair")[info.layout]
    launches_per_step = 1 if info.layout == 0 else 2
    traffic = committed_traffic(args.storage, chosen_layout)

    # end to end through the public API with host buffers: upload the state from
    # pinned host memory, advance, read the macroscopics back
    import numpy as np
    pops_host = torch.empty(Q * N, dtype=torch.float32).pin_memory()
    pops_host.copy_(torch.from_numpy(sim.populations().ravel()))
    ux_host = torch.empty(4 * N, dtype=torch.float32).pin_memory()
    import ctypes
    lib = vlbm.lib()
    F = ctypes.POINTER(ctypes.c_float)
    pp = ctypes.cast(pops_host.data_ptr(), F)
    outs = [ctypes.cast(ux_host.data_ptr() + k * N * 4, F) for k in range(4)]
    e2e_steps = args.e2e_steps
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    st = lib.vlbm_set_populations(sim.handle, pp, Q * N)
    st |= lib.vlbm_step(sim.handle, e2e_steps)
    st |= lib.vlbm_get_macroscopics(sim.handle, outs[0], outs[1], outs[2], outs[3], None)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    if st != 0:
        raise RuntimeError("e2e leg failed: " + lib.vlbm_last_error().decode())
    e2e_mlups = world * N * e2e_steps / e2e_s / 1e6
    h2d = Q * N * 4 / e2e_steps
    d2h = 4 * N * 4 / e2e_steps
    sim.sync()

    base = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        base = cpu_baseline()
    cube = None
    if rank == 0 and world == 1 and not args.no_cube:
        cube = cube_leg(vlbm, torch, local)
    cavity = None
    if rank == 0 and world == 1 and not args.no_cavity:
        cavity = cavity_leg(vlbm, torch, local)
    ibm_run = None
    if rank == 0 and world == 1 and not args.no_ibm:
        ibm_run = ibm_leg(vlbm, torch, local, steps=args.ibm_steps)
    serving = None
    if rank == 0 and world == 1 and not args.no_serving:
        serving = serving_leg(vlbm, args.serving_requests, args.serving_step_scale, args.serving_rate,
                              plain_repeats=args.serving_plain_repeats)

    if rank == 0:
        dtype = {"f32": "f32", "f16": "f32 arithmetic, f16 storage", "bf16": "f32 arithmetic, bf16 storage"}
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": dtype[args.storage], "data": "synthetic",
            "config": dict(config_dict(args.storage), layout=args.layout),
            "roofline": {"bound": "hbm", "achieved": achieved_gbs, "peak": peak, "unit": "GB/s",
                         "frac": achieved_gbs / peak, "traffic": traffic,
                         "peak_source": peak_kind,
                         "algorithmic_bytes_per_node": bytes_per_node,
                         "roofline_mlups": peak * 1e9 / bytes_per_node / 1e6},
            "cpu_baseline": base,
            "e2e": {"value": e2e_mlups, "unit": METRIC, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "note": "vlbm_set_populations from pinned host + K steps + vlbm_get_macroscopics to host, "
                            "wall clock, bytes amortised over K steps"},
            "gpu_launches": args.steps * launches_per_step,
            "kernel_variant": variant,
            "layout": ("natural", "zpair", "zpair_blocked")[info.layout],
            "clocks": clk,
            "lattice_256": cube,
            "powerlaw_cavity_256": cavity,
            "ibm_64_spheres": ibm_run,
            "serving": serving,
        }
        print(json.dumps(line), flush=True)
    sim.close()
    if dist:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
