#!/usr/bin/env python
"""Throughput of the per-timestep DEM path on B200: particle-steps/s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl xdem|reference]
                    [--workload NAME] [--n PARTICLES]

One step = one time step of the whole particle system (the reference's
takeTimeStep).  The default workload is a Lees-Edwards shear of ellipses at
the shapes of the learned-warm-start configuration (a/b ~ U[1,3], b in
{0.5, 0.7}, solid fraction 0.85, shear rate 1e-3 sqrt(kn/m_min)), 1,048,576
particles, plain FP64 closest-approach contact law.  The packing is generated
(RSA of bounding discs, then strain-controlled compression on the GPU) before
any timing.

Timed regions (all after W untimed warm-up steps, each of K steps):
  value      device time of K steps through xdem_run (CUDA events on the
             library's stream), inputs resident in HBM (state + contact
             history exceed the 126 MB L2);
  roofline   the same K steps with per-kernel CUDA events, dominant kernel;
  e2e        K x (upload state from pinned host memory, one step, download
             state), CUDA events on the library's stream.
The CPU baseline runs the compiled reference (oracle/_ref) with all host
threads on the same packing for a bounded number of steps.

Multi-GPU: the path does not shard (one system per GPU); with N ranks every
rank runs its own replica (weak scaling), value = sum over ranks.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

RANK = int(os.environ.get("RANK", "0"))
WORLD = int(os.environ.get("WORLD_SIZE", "1"))
LOCAL = int(os.environ.get("LOCAL_RANK", "0"))
if WORLD > 1:
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    devs = vis.split(",") if vis else [str(i) for i in range(64)]
    os.environ["CUDA_VISIBLE_DEVICES"] = devs[LOCAL]

import ctypes as C  # noqa: E402

import numpy as np  # noqa: E402

METRIC = "particle-steps/s, 1 B200: learned/batched FP32 vs plain FP64 GPU, same accuracy"
UNIT = "particle-steps/s"


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ---------------------------------------------------------------------------
# workloads
# ---------------------------------------------------------------------------
def config_le_ellipses(n):
    """The workload's description, the same in both arms (values that depend
    on the random sample are reported beside it, in workload_numbers)."""
    return {"workload": f"lees_edwards_shear_ellipses_{n}", "n_particles": n,
            "world": "LeesEdwardsBoundaryWorld",
            "contact_law": "closest approach (Zheng-Palffy-Muhoray quartic, Newton)",
            "aspect_ratio": "U[1,3]", "b": "{0.5,0.7}", "solid_fraction": 0.85,
            "shear_rate": "1e-3*sqrt(kn/m_min)", "dt": "0.02*sqrt(m_min/kn)",
            "l2": "inputs larger than L2 (state + contact history resident in HBM)"}


def workload_le_ellipses(n, seed):
    """Lees-Edwards shear of ellipses, a/b ~ U[1,3], b in {0.5,0.7}, phi 0.85."""
    from xdem_b200 import abi, inputs, packing
    from xdem_b200.world import make_control, make_params
    p, box = inputs.ellipse_system(n, b=inputs.c2_b, aspect=inputs.c4_aspect, phi_rsa_circle=0.40,
                                   phi=None, seed=seed)
    dt = inputs.time_step(p)
    m_min = float(np.min(p["mass"]))
    rate = 1e-3 * math.sqrt(inputs.KN / m_min)
    t = time.time()
    q, contacts, b, info = packing.compress(p, box, 0.85, dt, steps=4000, relax=2000)
    log(f"setup: compressed phi {info['phi0']:.3f} -> {info['phi']:.4f} in {info['steps']} steps "
        f"+ {info['relax']} relaxation steps, {time.time() - t:.1f}s, "
        f"{info['capped_newton']} non-terminating Newton solves")
    prm = make_params(abi.WORLD_LEES_EDWARDS, dt, b, inputs.KN, inputs.KT, inputs.RESTITUTION,
                      inputs.FRICTION, shift_strain_rate=rate)
    return {"particles": q, "contacts": contacts, "params": prm, "control": make_control(),
            # the compiled reference's Newton loop (EllipticParticle.cpp:621) has no
            # iteration cap and never returns on the few deeply overlapping pairs of
            # this packing that cycle, so the full-size CPU leg runs the C
            # restatement, identical but for stopping those
            "cpu_kind": "port",
            "cpu_note": "C restatement of the reference (it stops the Newton iterations the "
                        "compiled reference never returns from)",
            "config": config_le_ellipses(n),
            "numbers": {"solid_fraction_reached": round(info["phi"], 5), "shear_rate": rate,
                        "dt": dt}}


def train_warm_start(seed, n=262144, target_pairs=10_000_000, epochs=12):
    """The warm-start network of the learned configuration: pairs harvested
    from a Lees-Edwards shear of n ellipses with a/b ~ U[1,2], b in {0.5, 0.7},
    solid fraction 0.85 and shear rate 1e-3 sqrt(kn/m_min), trained on the GPU
    by the library's own kernels."""
    from xdem_b200 import abi, inputs, packing
    from xdem_b200.learned import Mlp
    from xdem_b200.world import World, make_control, make_params
    t0 = time.time()
    p, box = inputs.ellipse_system(n, b=inputs.c2_b, aspect=inputs.c2_aspect, phi_rsa_circle=0.40,
                                   phi=None, seed=seed + 100)
    dt = inputs.time_step(p)
    rate = 1e-3 * math.sqrt(inputs.KN / float(np.min(p["mass"])))
    q, contacts, b, _ = packing.compress(p, box, 0.85, dt, steps=4000, relax=1000)
    prm = make_params(abi.WORLD_LEES_EDWARDS, dt, b, inputs.KN, inputs.KT, inputs.RESTITUTION,
                      inputs.FRICTION, shift_strain_rate=rate)
    w = World(prm)
    w.raise_mask = ~abi.ERR_NEWTON
    w.set_particles(q)
    w.set_contacts(contacts)
    net = Mlp(seed=seed + 7)
    steps = 0
    while net.dataset_size() < target_pairs and steps < 2000:
        w.run(10, make_control())
        steps += 10
        net.harvest(w, stride=1, max_new=target_pairs - net.dataset_size())
    w.close()
    t1 = time.time()
    losses = net.train(epochs, batch=8192, lr=2e-3, seed=seed)
    t2 = time.time()
    info = {"harvest": f"LeesEdwardsBoundaryWorld shear of {n} ellipses, a/b U[1,2], phi 0.85, "
                       f"{steps} steps",
            "pairs": net.dataset_size(), "epochs": epochs, "batch": 8192,
            "loss_first_epoch": float(losses[0]), "loss_last_epoch": float(losses[-1]),
            "harvest_s": round(t1 - t0, 1), "train_s": round(t2 - t1, 1)}
    log(f"warm start: {info}")
    return net, info


def config_periodic_discs(n):
    return {"workload": f"periodic_discs_{n}", "n_particles": n, "world": "PeriodicBoundaryWorld",
            "contact_law": "disc-disc", "radii": "{0.5,0.7}", "solid_fraction": 0.70,
            "dt": "0.02*sqrt(m_min/kn)"}


def workload_periodic_discs(n, seed):
    """Bidisperse discs r 0.5/0.7 at phi 0.70, PeriodicBoundaryWorld (config-0 recipe at size n)."""
    from xdem_b200 import abi, inputs
    from xdem_b200.world import make_control, make_params
    p, box = inputs.disc_system(n, phi=0.70, seed=seed)
    dt = inputs.time_step(p)
    prm = make_params(abi.WORLD_PERIODIC, dt, box, inputs.KN, inputs.KT, inputs.RESTITUTION,
                      inputs.FRICTION)
    return {"particles": p, "contacts": None, "params": prm, "control": make_control(),
            "cpu_kind": "reference", "cpu_note": "compiled reference sources (oracle/_ref)",
            "config": config_periodic_discs(n), "numbers": {"dt": dt}}


def workload_batch_ensemble(n_systems, seed):
    """Batched uneven ensemble: n_systems independent PeriodicBoundaryWorld
    packings, N log-uniform in [1,000, 50,000] particles, solid fraction
    U[0.6, 0.8]; 40 % bidisperse discs (r 0.5/0.7), 40 % ellipses (a/b ~
    U[1,2], b in {0.5, 0.7}), 20 % clumps of 2-5 sub-discs.  Each packing is
    made by RSA and strain-controlled compression on the GPU."""
    from xdem_b200 import abi, inputs, packing
    from xdem_b200.world import make_control, make_params
    rng = np.random.default_rng(seed)
    kinds = (["disc"] * int(round(0.4 * n_systems)) + ["ellipse"] * int(round(0.4 * n_systems)))
    kinds += ["clump"] * (n_systems - len(kinds))
    kinds = [kinds[i] for i in rng.permutation(n_systems)]
    systems = []
    t = time.time()
    for s, kind in enumerate(kinds):
        N = int(round(math.exp(rng.uniform(math.log(1000), math.log(50000)))))
        phi = float(rng.uniform(0.6, 0.8))
        if kind == "disc":
            p, box = inputs.disc_system(N, phi_rsa=0.45, phi=None, seed=seed * 1000 + s)
        elif kind == "ellipse":
            p, box = inputs.ellipse_system(N, b=inputs.c2_b, aspect=inputs.c2_aspect,
                                           phi_rsa_circle=0.40, phi=None, seed=seed * 1000 + s,
                                           vel_sigma=0.01)
        else:
            p, box = inputs.clump_system(max(2, int(N / 4.5)), seed=seed * 1000 + s)
        dt = inputs.time_step(p)
        q, contacts, b, info = packing.compress(p, box, phi, dt, steps=1500, relax=500)
        systems.append({"particles": q, "contacts": contacts, "box": b, "dt": dt, "kind": kind,
                        "phi": info["phi"]})
    n = sum(len(sy["particles"]["x"]) for sy in systems)
    log(f"setup: {n_systems} systems, {n} particles, compressed in {time.time() - t:.1f}s")
    prm = make_params(abi.WORLD_PERIODIC, systems[0]["dt"], systems[0]["box"], inputs.KN, inputs.KT,
                      inputs.RESTITUTION, inputs.FRICTION)
    counts = {k: kinds.count(k) for k in ("disc", "ellipse", "clump")}
    return {"systems": systems, "params": prm, "control": make_control(),
            # ellipse systems hold pairs on which the compiled reference's uncapped
            # Newton loop does not return; the C restatement times the CPU leg
            "cpu_kind": "port",
            "cpu_note": "C restatement of the reference on the first systems of the batch "
                        "(capped Newton; the compiled reference does not return on the "
                        "ellipse systems' cycling Newton pairs)",
            "config": {"workload": f"batch_ensemble_{n_systems}x", "n_systems": n_systems,
                       "n_particles": n, "world": "PeriodicBoundaryWorld (batched)",
                       "system_kinds": counts, "particles_per_system": "log-uniform [1000, 50000]",
                       "solid_fraction": "U[0.6, 0.8]"}}


def cpu_sample_le_ellipses(n_sample, seed, threads):
    """A bounded sample of the Lees-Edwards ellipse shear made on the CPU only
    (no product library): n_sample ellipses of the workload's shapes, RSA,
    compression to solid fraction 0.85 by the C restatement, and the
    workload's shear rate."""
    import oracle
    from xdem_b200 import abi, inputs
    from xdem_b200.world import make_control, make_params
    q, contacts, box, dt = oracle.ellipse_sample(n_sample, seed, threads=threads, steps=2500,
                                                 relax=800)
    rate = 1e-3 * math.sqrt(inputs.KN / float(np.min(q["mass"])))
    prm = make_params(abi.WORLD_LEES_EDWARDS, dt, box, inputs.KN, inputs.KT, inputs.RESTITUTION,
                      inputs.FRICTION, shift_strain_rate=rate)
    return {"particles": q, "contacts": contacts, "params": prm, "control": make_control(),
            "cpu_kind": "reference",
            "cpu_note": f"{n_sample}-ellipse sample of the workload made on the CPU (RSA, C "
                        f"restatement compression to 0.85, same shapes and shear rate)"}


def cpu_sample_c0(seed, threads, n=1024):
    """The disc configuration on the CPU only: n bidisperse discs (r 0.5/0.7,
    50:50), RSA at 0.50, the C restatement's strain control to 0.70 and a
    relaxation, velocities N(0, 0.01^2), PeriodicBoundaryWorld."""
    import oracle
    from xdem_b200 import abi, inputs
    from xdem_b200.world import make_control, make_params
    rng = np.random.default_rng(seed)
    r = np.where(rng.permutation(n) < n // 2, 0.5, 0.7).astype(np.float64)
    box = inputs.box_for(float(np.sum(np.pi * r * r)), 0.50)
    x, y = oracle.rsa_discs(r, box, seed + 1)
    shape = np.zeros(n, np.int32)
    zero = np.zeros(n)
    p = {"shape": shape, "up_level": np.arange(n, dtype=np.int32), "setting": np.zeros(n, np.int32),
         "is_rattler": np.zeros(n, np.int32), "outer_radius": r, "radius": r.copy(),
         "aspect_ratio": np.ones(n), "x": x, "y": y, "vx": zero.copy(), "vy": zero.copy(),
         "rot": zero.copy(), "rot_vel": zero.copy()}
    p.update(oracle.particle_properties(shape, r, np.ones(n)))
    dt = 0.02 * math.sqrt(float(np.min(p["mass"])) / inputs.KN)
    q, _, box = oracle.strain_compress(oracle.PortWorld, p, box, dt, 0.70, 2000, 500,
                                       threads=threads)
    q["vx"] = rng.normal(0.0, 0.01, n)
    q["vy"] = rng.normal(0.0, 0.01, n)
    q["rot_vel"] = np.zeros(n)
    prm = make_params(abi.WORLD_PERIODIC, dt, box, inputs.KN, inputs.KT, inputs.RESTITUTION,
                      inputs.FRICTION)
    return {"particles": q, "contacts": None, "params": prm, "control": make_control(),
            "cpu_kind": "reference", "cpu_note": f"{n} discs at 0.70 made on the CPU"}


def cpu_sample_c1_prefix(steps=4000):
    """The ellipse compression's start (tests/golden/long_c1_closest.npz: 512
    ellipses, b ~ U[0.4, 0.6], a = 1.5 b, an overlap-free RSA at 0.50, strain
    control at -1e-4), over a prefix on which the compiled reference returns
    (it stops returning after ~10,000 steps of this run)."""
    from xdem_b200 import abi, inputs
    from xdem_b200.world import make_control, make_params
    z = np.load(os.path.join(ROOT, "tests", "golden", "long_c1_closest.npz"))
    p = {k[2:]: z[k] for k in z.files if k.startswith("p_")}
    prm = make_params(abi.WORLD_PERIODIC_CONTROL, float(z["dt"]), z["box0"], inputs.KN, inputs.KT,
                      inputs.RESTITUTION, inputs.FRICTION)
    rate = float(z["rate"])
    return {"particles": p, "contacts": None, "params": prm, "steps": steps,
            "control": make_control(update_stress=True, box_law=abi.BOX_STRAIN, p0=rate, p1=rate),
            "cpu_kind": "reference", "cpu_note": "512-ellipse compression prefix"}


def reference_vs_restatement(threads, seed):
    """Speed of the compiled reference and of the C restatement on the same
    CPU-made inputs where the reference returns: the disc configuration
    (1,024 discs, `threads` threads each) and the first steps of the ellipse
    compression (512 ellipses, one thread each).  The restatement is what the
    full-size CPU leg times; this relates it to the reference's own code."""
    out = {}
    cases = (("discs_1024", lambda: cpu_sample_c0(seed, threads), threads),
             ("ellipses_512_compression", cpu_sample_c1_prefix, 1))
    for name, make, th in cases:
        work = make()
        steps = work.get("steps", 400)
        ref = run_cpu(work, steps, 1, th, budget_s=8.0, timeout_s=120, kind="reference")
        port = run_cpu(work, steps, 1, th, budget_s=8.0, timeout_s=120, kind="port")
        entry = {"threads": th, "reference": ref.get("value"), "restatement": port.get("value")}
        if ref.get("kind") != "reference" or "error" in ref:
            entry["reference_note"] = ref.get("error", "compiled reference not available")
        if entry["reference"] and entry["restatement"]:
            entry["restatement_over_reference"] = entry["restatement"] / entry["reference"]
        out[name] = entry
    return out


WORKLOADS = {"le_ellipses": workload_le_ellipses, "periodic_discs": workload_periodic_discs,
             "batch_ensemble": workload_batch_ensemble}


# ---------------------------------------------------------------------------
# measurement helpers
# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during a timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index=0):
        self.index = index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 8:
                self.rows.append(parts)

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[4 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic_per_particle(kernel):
    """DRAM bytes per particle of `kernel` from the committed ncu summary, or None."""
    path = os.path.join(ROOT, "profiles", "traffic_per_particle.txt")
    if not os.path.exists(path):
        return None
    for line in open(path):
        parts = line.split()
        if len(parts) >= 2 and parts[0] == kernel:
            try:
                return float(parts[1])
            except ValueError:
                return None
    return None


def kernel_bytes(kernel, n, contacts, pairs, entries=0):
    """Algorithmic DRAM bytes of one launch of a contact-update kernel, with
    every particle's data counted once (neighbour re-reads hit L2).
    k_candidates (with candidate lists): per particle the owner's data
      (position 16, radius 8, outer radius 8, axis record 16, setting 4,
      up-level 4, cell 4, list length 4, old record count 4 and first
      record 4) = 72 B, written: its record count and first record 8 B =
      80 B (the binning kernel writes the body record); per list entry 4 B;
      per old contact its partner's id and memory position 8 B; per listed
      pair a 16 B entry.
    k_pair_forces: per particle the state the geometry reads (position 16,
      velocity 16, orientation 8, spin 8, radius 8, aspect 8, outer radius 8,
      shape 4, mass 8, setting 4, id 4) = 92 B; per listed pair its entry 16 B;
      per contact the previous history (partner 4, normal 16, shear 16,
      damping 8 = 44 B) and the new record (partner 4, normal 16, shear 16,
      damping 8, force 16, torques 16, branch vector 16 = 92 B); per listed
      pair that does not touch, an empty-slot mark (4 B)."""
    if kernel == "k_candidates":
        return 80.0 * n + 4.0 * entries + 8.0 * contacts + 16.0 * pairs
    return 92.0 * n + 16.0 * pairs + 136.0 * contacts + 4.0 * max(pairs - contacts, 0)


def _cpu_child(paths, steps, warmup, threads, budget_s, kind):
    """Child process: times the compiled reference (kind "reference") or the
    C restatement (kind "port") on the systems saved at `paths` (each stepped
    in turn, the same number of steps); prints one JSON line."""
    import oracle
    from xdem_b200 import abi
    if kind == "reference" and not oracle.ref_available():
        kind = "port"
    W = oracle.RefWorld if kind == "reference" else oracle.PortWorld
    worlds, sizes = [], []
    ctl = abi.Control()
    for path in paths.split(","):
        z = np.load(path, allow_pickle=False)
        p = {k[2:]: z[k] for k in z.files if k.startswith("p_")}
        c = {k[2:]: z[k] for k in z.files if k.startswith("c_")}
        prm = abi.Params()
        C.memmove(C.byref(prm), z["params"].tobytes(), C.sizeof(abi.Params))
        prm.precision = abi.PRECISION_FP64
        C.memmove(C.byref(ctl), z["control"].tobytes(), C.sizeof(abi.Control))
        w = W(prm, threads)
        w.raise_mask = ~abi.ERR_NEWTON
        w.set_particles(p)
        if c and len(c["id_i"]):
            w.set_contacts(c)
        worlds.append(w)
        sizes.append(len(p["x"]))
    for _ in range(warmup):
        for w in worlds:
            w.run(1, ctl)
    t0 = time.perf_counter()
    for w in worlds:
        w.run(1, ctl)
    one = time.perf_counter() - t0
    k = max(1, min(steps, int(budget_s / max(one, 1e-6))))
    t0 = time.perf_counter()
    for w in worlds:
        w.run(k, ctl)
    dt = time.perf_counter() - t0
    n = sum(sizes)
    print(json.dumps({"value": n * k / dt, "steps": k, "kind": kind, "one_step_s": one,
                      "systems": len(worlds), "particles": n}), flush=True)


def _system_params(work, sy):
    """World parameters of one system of a batch workload."""
    from xdem_b200 import abi
    prm = abi.Params()
    C.memmove(C.byref(prm), C.byref(work["params"]), C.sizeof(abi.Params))
    prm.xmin, prm.xmax, prm.ymin, prm.ymax = (float(v) for v in sy["box"])
    prm.dt = sy["dt"]
    return prm


def run_cpu(work, steps, warmup, threads, budget_s=25.0, timeout_s=300, max_particles=150000,
            kind=None):
    """Times the CPU implementation named by `kind` (default work["cpu_kind"])
    in a child process with a watchdog (a batch: its first systems, up to
    max_particles).  Returns the child's result dict or {"error": ...}."""
    kind = kind or work["cpu_kind"]
    import tempfile
    if "systems" in work:
        items, total = [], 0
        for sy in work["systems"]:
            if items and total + len(sy["particles"]["x"]) > max_particles:
                break
            items.append((sy["particles"], sy["contacts"], _system_params(work, sy)))
            total += len(sy["particles"]["x"])
    else:
        items = [(work["particles"], work["contacts"], work["params"])]
    paths = []
    for k, (p, c, prm) in enumerate(items):
        path = os.path.join(tempfile.gettempdir(), f"xdem_bench_{os.getpid()}_{k}.npz")
        arrs = {f"p_{key}": v for key, v in p.items() if isinstance(v, np.ndarray)}
        if c is not None:
            arrs.update({f"c_{key}": v for key, v in c.items()})
        arrs["params"] = np.frombuffer(bytes(prm), np.uint8)
        arrs["control"] = np.frombuffer(bytes(work["control"]), np.uint8)
        np.savez(path, **arrs)
        paths.append(path)
    path = ",".join(paths)
    cmd = [sys.executable, os.path.abspath(__file__), "--cpu-child", path, "--steps", str(steps),
           "--warmup", str(warmup), "--threads", str(threads), "--budget", str(budget_s),
           "--cpu-kind", kind]
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    try:
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout_s, env=env)
        lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
        if r.returncode != 0 or not lines:
            return {"error": f"exit {r.returncode}: {r.stderr.strip()[-300:]}"}
        return json.loads(lines[-1])
    except subprocess.TimeoutExpired:
        return {"error": f"no result within {timeout_s} s"}
    finally:
        for p_ in paths:
            if os.path.exists(p_):
                os.remove(p_)


def batch_contacts(systems, first):
    """The systems' contact histories with ids made global."""
    keys = systems[0]["contacts"].keys()
    out = {}
    for key in keys:
        parts = []
        for sy, f in zip(systems, first):
            v = sy["contacts"][key]
            parts.append(v + f if key in ("id_i", "id_j") else v)
        out[key] = np.ascontiguousarray(np.concatenate(parts))
    return out


def measure_loop(work, precision, args):
    """The batch workload as a per-system loop: one world per system on one
    stream, each run for the K steps in turn (CUDA events around the loop)."""
    from xdem_b200 import abi
    from xdem_b200.world import World
    worlds = []
    for sy in work["systems"]:
        prm = _system_params(work, sy)
        prm.precision = precision
        w = World(prm)
        w.raise_mask = ~(abi.ERR_NEWTON | abi.ERR_NONFINITE)
        w.set_particles(sy["particles"])
        w.set_contacts(sy["contacts"])
        worlds.append(w)
    lib = worlds[0].lib
    stream = C.c_void_p(0)
    lib.xdem_get_stream(worlds[0].h, C.byref(stream))
    for w in worlds[1:]:
        lib.xdem_set_stream(w.h, stream)
    ctl = work["control"]
    for w in worlds:
        w.run(max(args.warmup, 3), ctl)
    n = sum(len(sy["particles"]["x"]) for sy in work["systems"])
    worlds[0].synchronize()
    lib.xdem_timer_start(worlds[0].h)
    for w in worlds:
        w.run(args.steps, ctl)
    ms = C.c_double(0.0)
    lib.xdem_timer_stop(worlds[0].h, C.byref(ms))
    for w in worlds[1:]:
        lib.xdem_set_stream(w.h, None)
    for w in reversed(worlds):
        w.close()
    return {"value": n * args.steps / (ms.value / 1e3), "ms_per_step": ms.value / args.steps}


def measure(work, precision, args, dist, full=True, net=None, kernels=False):
    """Times `args.steps` steps of the workload at the given precision.
    full: also the per-kernel roofline pass and the end-to-end pass;
    kernels: (without full) the per-kernel pass alone;
    net: the learned warm start to attach."""
    from xdem_b200 import abi
    from xdem_b200.learned import warm_stats
    from xdem_b200.world import World

    prm = abi.Params()
    C.memmove(C.byref(prm), C.byref(work["params"]), C.sizeof(abi.Params))
    prm.precision = precision
    w = World(prm)
    # capped Newton solves are counted and reported, not raised; so is a
    # non-finite state (the reference's closest-approach arithmetic can make
    # one, and the reference runs on through it): both show in `status`
    w.raise_mask = ~(abi.ERR_NEWTON | abi.ERR_NONFINITE)
    if "systems" in work:
        systems = work["systems"]
        w.set_batch([sy["particles"] for sy in systems], [sy["box"] for sy in systems],
                    [sy["dt"] for sy in systems])
        _, first = w.batch_info()
        w.set_contacts(batch_contacts(systems, first))
        n = int(first[-1])
    else:
        p = work["particles"]
        n = len(p["x"])
        w.set_particles(p)
        if work["contacts"] is not None and len(work["contacts"]["id_i"]):
            w.set_contacts(work["contacts"])
    ctl = work["control"]
    lib = w.lib
    if net is not None:
        net.attach(w)

    def barrier():
        if dist:
            dist.barrier()

    def max_over_ranks(v):
        if not dist:
            return v
        import torch
        t = torch.tensor([v], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    w.run(max(args.warmup, 3), ctl)

    # ---- value: device time of K steps, repeated ---------------------------
    # Each repeat times exactly K steps (CUDA events on the library's stream,
    # a barrier and a synchronisation on both sides); the repeats continue
    # until they cover a second of device time (at least five), so that the
    # clock sampler (every 100 ms) sees the timed region; the value is the
    # median repeat.
    clocks = ClockSampler(0)
    w.reset_newton_stats()
    clocks.start()
    reps, launches, done_total = [], 0, 0
    while len(reps) < 5 or (sum(reps) < 1000.0 and len(reps) < 400):
        barrier()
        w.synchronize()
        l0 = w.launch_count()
        lib.xdem_range_push(b"bench_value")
        lib.xdem_timer_start(w.h)
        done = w.run(args.steps, ctl)
        ms = C.c_double(0.0)
        lib.xdem_timer_stop(w.h, C.byref(ms))
        lib.xdem_range_pop()
        launches = w.launch_count() - l0
        done_total += done
        reps.append(max_over_ranks(ms.value))
    clk = clocks.stop()
    ms_total = statistics.median(reps)
    contacts = w.count_contacts()
    solves, iters, capped = w.newton_stats()
    out = {"value": n * done * WORLD / (ms_total / 1e3), "ms_per_step": ms_total / max(done, 1),
           "done": done, "contacts": contacts, "launches": int(launches), "clocks": clk,
           "repeats": {"count": len(reps), "ms_min": min(reps), "ms_median": ms_total,
                       "ms_max": max(reps)},
           "newton": {"solves_per_step": solves / max(done_total, 1),
                      "iterations_per_solve": iters / max(solves, 1),
                      "nonterminating_solves_per_step": capped / max(done_total, 1)}}
    lists = w.candidate_list_stats()
    if lists["capacity"] > 0:
        out["candidate_lists"] = {"builds_per_step": lists["builds"] / max(done_total, 1),
                                  "entries_per_particle": lists["entries"] / n,
                                  "longest": lists["longest"], "capacity": lists["capacity"]}
    if net is not None:
        ws = warm_stats(w)
        off = max(ws["offered"], 1)
        out["warm_start"] = {"offered_per_step": ws["offered"] / max(done, 1),
                             "used_fraction": ws["used"] / off,
                             "fallback_fraction": (ws["rejected"] + ws["restarted"]) / off,
                             "contact_logit_accuracy": ws["logit_right"] / off}
    if not full:
        if kernels:
            w.set_profiling(True)
            w.run(args.steps, ctl)
            prof = w.profile()
            w.set_profiling(False)
            out["kernel_ms_per_step"] = {k: round(v[1] / args.steps, 5) for k, v in prof.items()}
            out["pairs_per_step"] = w.pair_count()
        out["status"] = w.synchronize()
        w.close()
        return out

    # ---- roofline: per-kernel events over the same number of steps ---------
    w.set_profiling(True)
    w.run(args.steps, ctl)
    prof = w.profile()
    w.set_profiling(False)
    pairs = w.pair_count()
    kname = max(("k_candidates", "k_pair_forces"), key=lambda k: prof.get(k, (1, 0.0))[1])
    upd = prof[kname]
    avg_s = upd[1] / upd[0] / 1e3
    lists = w.candidate_list_stats()
    alg_bytes = kernel_bytes(kname, n, contacts, pairs, lists["entries"])
    peak, peak_kind = measured_peaks()
    achieved = alg_bytes / avg_s / 1e9
    traffic_pp = ncu_traffic_per_particle(kname)
    total = sum(x[1] for x in prof.values())
    out["roofline"] = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                       "frac": achieved / peak, "peak_source": peak_kind,
                       "kernel": kname, "algorithmic_bytes_per_launch": alg_bytes,
                       "pairs_per_step": pairs, "avg_launch_ms": avg_s * 1e3,
                       "traffic": None if traffic_pp is None else traffic_pp * n}
    out["kernel_share"] = {k: round(v[1] / total, 4) for k, v in prof.items()}
    out["kernel_ms_per_step"] = {k: round(v[1] / args.steps, 5) for k, v in prof.items()}
    out["profiled_ms_per_step"] = total / args.steps

    # ---- e2e through the C-ABI with pinned host buffers ----------------------
    nbytes = 8 * n
    bufs = [lib.xdem_host_alloc(nbytes) for _ in range(6)]
    if not all(bufs):
        raise RuntimeError("xdem_host_alloc failed")
    st = w.get_state()
    for buf, key in zip(bufs, ("x", "y", "vx", "vy", "rot", "rot_vel")):
        C.memmove(buf, st[key].ctypes.data, nbytes)
    one = abi.Control()
    C.memmove(C.byref(one), C.byref(ctl), C.sizeof(abi.Control))
    done_c = C.c_int32(0)
    barrier()
    w.synchronize()
    lib.xdem_timer_start(w.h)
    for _ in range(args.steps):
        lib.xdem_upload_state(w.h, *[C.cast(b, C.POINTER(C.c_double)) for b in bufs])
        lib.xdem_run(w.h, 1, C.byref(one), C.byref(done_c))
        lib.xdem_download_state(w.h, *[C.cast(b, C.POINTER(C.c_double)) for b in bufs])
    ms_e2e = C.c_double(0.0)
    lib.xdem_timer_stop(w.h, C.byref(ms_e2e))
    e2e_ms = max_over_ranks(ms_e2e.value)
    for b in bufs:
        lib.xdem_host_free(b)
    out["e2e"] = {"value": n * args.steps * WORLD / (e2e_ms / 1e3), "unit": UNIT,
                  "h2d_bytes_per_step": 6 * nbytes, "d2h_bytes_per_step": 6 * nbytes}
    out["status"] = w.synchronize()
    w.close()
    return out


def accuracy(work, steps=2000, sample_every=100, short=20):
    """Mixed precision against FP64 on the workload's packing: (1) one step
    from the same state and history, the largest per-contact force difference
    over the largest FP64 contact force (bar 1e-5); (2) the shear stress (xy)
    of that step (bar 1e-6) and the largest relative difference over the
    first `short` steps; (3) the mean shear stress over `steps` further
    steps, sampled every `sample_every` steps, and its relative difference
    (bar 0.5 %).  (2) and (3) are given beside the same differences between
    the FP64 path and an FP64 twin started from positions scaled by
    (1 + 1e-15): a few deep contacts whose closest-approach root changes with
    the last bit of the inputs come and go within a few steps in either
    pair, which sets the floor of (3).  The FP64 path is the one the parity
    tests pin to the reference (1e-10 per contact)."""
    from xdem_b200 import abi
    from xdem_b200.world import World, make_control

    def world(prec, scale_x=1.0):
        prm = abi.Params()
        C.memmove(C.byref(prm), C.byref(work["params"]), C.sizeof(abi.Params))
        prm.precision = prec
        w = World(prm)
        w.raise_mask = ~abi.ERR_NEWTON
        p = dict(work["particles"])
        if scale_x != 1.0:
            p["x"] = p["x"] * scale_x
        w.set_particles(p)
        if work["contacts"] is not None and len(work["contacts"]["id_i"]):
            w.set_contacts(work["contacts"])
        return w

    t0 = time.time()
    w64, wmx, wtw = (world(abi.PRECISION_FP64), world(abi.PRECISION_MIXED),
                     world(abi.PRECISION_FP64, 1.0 + 1e-15))
    worlds = (w64, wmx, wtw)
    ctl = make_control(update_stress=True)
    first = []
    for w in worlds:
        w.run(1, ctl)
        first.append(w.getStress()[1])
    c64, cmx = w64.get_contacts(), wmx.get_contacts()
    k64 = c64["id_i"].astype(np.int64) << 32 | c64["id_j"].astype(np.int64)
    kmx = cmx["id_i"].astype(np.int64) << 32 | cmx["id_j"].astype(np.int64)
    common, i64, imx = np.intersect1d(k64, kmx, assume_unique=True, return_indices=True)
    f64 = np.stack([c64["fn_x"] + c64["ft_x"], c64["fn_y"] + c64["ft_y"]], 1)
    fmx = np.stack([cmx["fn_x"] + cmx["ft_x"], cmx["fn_y"] + cmx["ft_y"]], 1)
    scale = float(np.max(np.hypot(f64[:, 0], f64[:, 1])))
    err = np.hypot(*(fmx[imx] - f64[i64]).T) / scale
    one_step = {"max_force_error": float(err.max()), "p99_99_force_error": float(np.quantile(err, 0.9999)),
                "contacts_over_1e-5": int(np.sum(err > 1e-5)), "contacts": int(len(k64)),
                "contacts_only_fp64": int(len(k64) - len(common)),
                "contacts_only_mixed": int(len(kmx) - len(common)), "bar": 1e-5}
    names = ("fp64", "mixed", "fp64_twin")
    # a world whose state turns non-finite (the reference's closest-approach
    # arithmetic can produce a NaN overlap) leaves the comparison, with the
    # step at which it did
    nonfinite = {}

    def advance(k, nsteps, done):
        if names[k] in nonfinite:
            return None
        try:
            worlds[k].run(nsteps, ctl)
        except abi.XdemError as e:
            nonfinite[names[k]] = f"step {done + nsteps}: {e}"
            return None
        return worlds[k].getStress()[1]

    per_step = [first]
    for i in range(1, short):
        per_step.append([advance(k, 1, i) for k in range(3)])

    def rel(a, b):
        return abs(a - b) / abs(b) if a is not None and b is not None else None

    def max_rel(k):
        v = [rel(r[k], r[0]) for r in per_step]
        return max(v) if v and all(x is not None for x in v) else None

    short_h = {"first_step_relative_difference_mixed": rel(first[1], first[0]),
               "first_step_relative_difference_fp64_twin": rel(first[2], first[0]),
               "bar": 1e-6, "steps": short, "max_relative_difference_mixed": max_rel(1),
               "max_relative_difference_fp64_twin": max_rel(2)}
    series = [[], [], []]
    for i in range(steps // sample_every):
        for k in range(3):
            v = advance(k, sample_every, short + i * sample_every)
            if v is not None:
                series[k].append(v)
    full_len = steps // sample_every
    m = [float(np.mean(s)) if len(s) == full_len else None for s in series]
    shear = {"steps": steps, "samples": full_len, "mean_shear_stress_fp64": m[0],
             "mean_shear_stress_mixed": m[1], "relative_difference": rel(m[1], m[0]),
             "mean_shear_stress_fp64_twin": m[2], "relative_difference_fp64_twin": rel(m[2], m[0]),
             "bar": 5e-3}
    if nonfinite:
        shear["nonfinite"] = nonfinite
    for w in worlds:
        w.close()
    log(f"accuracy: {one_step}, {short_h}, {shear}, {time.time() - t0:.1f}s")
    return {"one_step_forces": one_step, "short_horizon_shear_stress": short_h,
            "mean_shear_stress": shear}


def mlp_kernels():
    """A few launches of the learned warm start's kernels, for a profiler:
    training (k_mlp_train) on 262,144 synthetic samples, 2 epochs, then
    inference (k_mlp_warm) in a Lees-Edwards world of 65,536 ellipses
    (a/b ~ U[1,3], b in {0.5, 0.7}) with the network attached, 8 steps."""
    from xdem_b200 import abi, inputs
    from xdem_b200.learned import Mlp
    from xdem_b200.world import World, make_control, make_params
    net = Mlp(seed=3)
    rng = np.random.default_rng(0)
    n = 262144
    net.add_samples(rng.normal(0, 1, (n, 7)).astype(np.float32),
                    rng.uniform(0.5, 1.0, n).astype(np.float32),
                    (rng.uniform(0, 1, n) > 0.5).astype(np.float32))
    net.train(2, batch=8192, lr=1e-3, seed=1)
    p, box = inputs.ellipse_system(65536, b=inputs.c2_b, aspect=inputs.c4_aspect,
                                   phi_rsa_circle=0.40, phi=None, seed=5)
    area = (box[1] - box[0]) * (box[3] - box[2])
    box = inputs.scale_to_fraction(p, box, p["volume"].sum(), p["volume"].sum() / area * 1.6)
    prm = make_params(abi.WORLD_LEES_EDWARDS, inputs.time_step(p), box, inputs.KN, inputs.KT,
                      inputs.RESTITUTION, inputs.FRICTION, shift_strain_rate=0.1)
    w = World(prm)
    w.raise_mask = ~(abi.ERR_NEWTON | abi.ERR_NONFINITE)
    w.set_particles(p)
    net.attach(w)
    w.run(8, make_control())
    log(f"mlp kernels: {w.pair_count()} listed pairs in the last step")
    w.close()
    net.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="xdem", choices=["xdem", "reference"])
    ap.add_argument("--workload", default="le_ellipses", choices=sorted(WORKLOADS))
    ap.add_argument("--n", type=int, default=1 << 20)
    ap.add_argument("--systems", type=int, default=128, help="batch_ensemble: number of systems")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"],
                    help="arithmetic of the headline path (the other one is timed beside it)")
    ap.add_argument("--no-compare", action="store_true", help="skip the second precision")
    ap.add_argument("--no-learned", action="store_true",
                    help="skip training and timing the learned warm start")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--mlp-kernels", action="store_true",
                    help="only launch the learned warm start's kernels a few times (profiling)")
    ap.add_argument("--cpu-child", default=None, help=argparse.SUPPRESS)
    ap.add_argument("--cpu-kind", default="port", help=argparse.SUPPRESS)
    ap.add_argument("--threads", type=int, default=0, help=argparse.SUPPRESS)
    ap.add_argument("--budget", type=float, default=20.0, help=argparse.SUPPRESS)
    args = ap.parse_args()
    if args.mlp_kernels:
        mlp_kernels()
        return
    if args.cpu_child:
        _cpu_child(args.cpu_child, args.steps, args.warmup, args.threads or os.cpu_count(),
                   args.budget, args.cpu_kind)
        return

    dist = None
    if WORLD > 1:
        import torch
        import torch.distributed as dist_mod
        from datetime import timedelta
        dist_mod.init_process_group("gloo", timeout=timedelta(seconds=600))
        dist = dist_mod

    if args.impl == "reference":
        # The reference's CPU implementation of the path, on the host cores,
        # on a bounded sample of the workload built without the product
        # library: the compiled reference where it returns within the
        # watchdog, else the C restatement.
        if RANK != 0:
            if dist:
                dist.destroy_process_group()
            return
        threads = os.cpu_count() or 1
        if args.workload == "le_ellipses":
            work = cpu_sample_le_ellipses(4096, args.seed, threads)
            config = config_le_ellipses(args.n)
        elif args.workload == "periodic_discs":
            work = cpu_sample_c0(args.seed, threads, n=args.n)
            config = config_periodic_discs(args.n)
        else:
            work = WORKLOADS[args.workload](args.systems, args.seed)
            config = work["config"]
        config = dict(config, parallelism="single")
        res = run_cpu(work, args.steps, 1, threads, budget_s=40.0, timeout_s=150, kind="reference")
        if "error" in res:
            note = res["error"]
            res = run_cpu(work, args.steps, 1, threads, budget_s=40.0, timeout_s=150, kind="port")
            work["cpu_note"] += f"; the compiled reference gave no result ({note})"
        if "error" in res:
            print(json.dumps({"impl": "reference", "unavailable": res["error"]}), flush=True)
        else:
            v, k = res["value"], res["steps"]
            sample = (f"{k} steps of {res['particles']} particles in {res['systems']} system(s) "
                      f"after 1 warm-up step, {threads} threads; {work['cpu_note']}")
            line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT,
                    "n_gpus": args.gpus, "steps": k, "warmup": 1,
                    "ms_per_step": 1e3 * config["n_particles"] / v,
                    "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                    "data": "synthetic", "config": config,
                    "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": res["kind"],
                                     "sample": sample},
                    "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0,
                            "d2h_bytes_per_step": 0}}
            print(json.dumps(line), flush=True)
        if dist:
            dist.destroy_process_group()
        return

    from xdem_b200 import abi
    prec = {"mixed": abi.PRECISION_MIXED, "fp64": abi.PRECISION_FP64}
    other = "fp64" if args.precision == "mixed" else "mixed"

    size = args.n if args.workload != "batch_ensemble" else args.systems
    work = WORKLOADS[args.workload](size, args.seed + RANK)
    n = work["config"]["n_particles"]
    head = measure(work, prec[args.precision], args, dist, full=True)
    cmp_ = None if args.no_compare else measure(work, prec[other], args, dist, full=False,
                                                kernels=True)
    loop = None
    if "systems" in work:
        loop = measure_loop(work, prec[args.precision], args)
    learned = None
    if args.workload == "le_ellipses" and not args.no_learned and not args.no_compare:
        net, tinfo = train_warm_start(args.seed)
        learned = {"training": tinfo}
        for name, pr in (("fp64_warm", abi.PRECISION_FP64), ("mixed_warm", abi.PRECISION_MIXED)):
            r = measure(work, pr, args, dist, full=False, net=net, kernels=True)
            learned[name] = {"value": r["value"], "ms_per_step": r["ms_per_step"],
                             "newton": r["newton"], "warm_start": r["warm_start"],
                             "kernel_ms_per_step": r["kernel_ms_per_step"],
                             "pairs_per_step": r["pairs_per_step"],
                             "status": r["status"], "clocks": r["clocks"]}
        net.close()

    # ---- CPU baseline (rank 0, N = 1 only) ----------------------------------
    cpu = None
    if RANK == 0 and WORLD == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        res = run_cpu(work, 50, 1, threads, budget_s=20.0)
        if "error" in res:
            cpu = {"value": None, "unit": UNIT, "cores": threads, "kind": work["cpu_kind"],
                   "sample": res["error"]}
        else:
            cpu = {"value": res["value"], "unit": UNIT, "cores": threads, "kind": res["kind"],
                   "sample": f"{res['steps']} steps of {res['particles']} particles in "
                             f"{res['systems']} system(s) after 1 warm-up step "
                             f"({res['one_step_s']:.2f} s per step); {work['cpu_note']}"}

    acc = None
    if args.workload == "le_ellipses" and not args.no_compare and args.precision == "mixed":
        acc = accuracy(work)
    cpu_cmp = None
    if RANK == 0 and WORLD == 1 and not args.no_cpu_baseline:
        cpu_cmp = reference_vs_restatement(os.cpu_count() or 1, args.seed)
        if cpu is not None:
            cpu["reference_vs_restatement"] = cpu_cmp

    cfg = dict(work["config"])
    cfg.setdefault("l2", "inputs larger than L2 (state + contact history resident in HBM)")
    cfg["parallelism"] = f"replicas{WORLD}" if WORLD > 1 else "single"
    numbers = dict(work.get("numbers", {}))
    numbers["contacts"] = head["contacts"]
    line = {
        "metric": METRIC, "value": head["value"], "unit": UNIT, "n_gpus": WORLD,
        "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": head["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64" if args.precision == "mixed" else "f64",
        "data": "synthetic", "config": cfg, "precision": args.precision,
        "workload_numbers": numbers,
        "contacts_per_s": head["contacts"] * head["done"] * WORLD / (head["ms_per_step"] * head["done"] / 1e3),
        "e2e": head["e2e"], "gpu_launches": head["launches"], "roofline": head["roofline"],
        "kernel_share": head["kernel_share"], "kernel_ms_per_step": head["kernel_ms_per_step"],
        "profiled_ms_per_step": head["profiled_ms_per_step"],
        "clocks": head["clocks"], "repeats": head["repeats"], "status": head["status"],
        "newton": head["newton"], "cpu_baseline": cpu,
    }
    if acc is not None:
        line["accuracy_mixed_vs_fp64"] = acc
    if "candidate_lists" in head:
        line["candidate_lists"] = head["candidate_lists"]
    if loop is not None:
        line["per_system_loop"] = {"value": loop["value"], "ms_per_step": loop["ms_per_step"],
                                   "what": "one world per system, each run for the K steps in "
                                           "turn on one stream"}
        line["speedup_vs_per_system_loop"] = head["value"] / loop["value"]
    if learned is not None:
        line["learned"] = learned
    if cmp_ is not None:
        line[other] = {"value": cmp_["value"], "ms_per_step": cmp_["ms_per_step"],
                       "contacts": cmp_["contacts"], "newton": cmp_["newton"],
                       "kernel_ms_per_step": cmp_["kernel_ms_per_step"],
                       "clocks": cmp_["clocks"], "status": cmp_["status"]}
        line[f"speedup_vs_{other}"] = head["value"] / cmp_["value"]
    if RANK == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
