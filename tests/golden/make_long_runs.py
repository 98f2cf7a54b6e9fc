"""Generates the long-run golden fixtures in this folder from the COMPILED
REFERENCE (oracle/_ref/libxdem_ref.so, one thread), at the benchmark
configurations' shapes and sizes:

  long_c0_discs.npz
      1,024 bidisperse discs (r 0.5/0.7 50:50, density 1) in a
      PeriodicBoundaryWorld at solid fraction 0.70, velocities N(0, 0.01^2),
      zero spin, kn 1e4, kt 0.5 kn, damping ratio 0.3, friction 0.5,
      dt = 0.02 sqrt(m_min/kn), 10,000 FP64 steps.  The packing: random
      sequential addition at 0.50 (0.70 is beyond what RSA reaches), then the
      reference's own strain control (updatePeriodicBoundary_strainControl) to
      0.70 and a relaxation, after which velocities are drawn afresh and the
      run starts without contact history.  Sampled every 500 steps: the total
      stress (updateTotalStress), the contact count and the kinetic energy;
      at the end: the state, the contacts and QuadronAnalysis's rattler-free
      coordination number and solid fraction.
  long_c1_<law>.npz
      The isotropic compression of ellipses (b ~ U[0.4, 0.6], a = 1.5 b,
      orientations U[0, pi)) at a reduced size, by both ellipse laws: an
      overlap-free RSA of the ellipses themselves at solid fraction 0.50, then
      PeriodicControlWorld strain control at rate -1e-4 (the reference's
      convention, scale = 1 + rate L dt per step) until trace(stress)/2
      reaches 1e-3 kn = 10.  Recorded: the steps taken, the solid fraction
      and box at the stop, the stress sampled along the way, and the final
      Z and phi.

The disc fixture also holds the C restatement's (oracle/liboracle.so) run
and three reference runs whose initial velocities differ by one ulp.  The
compiled reference stops returning during the closest-approach compression
(a Newton iteration without end between steps 10,000 and 20,000), so that
fixture pins the restatement to the reference on the first 10,000 steps and
records the restatement's full run and two runs with one orientation moved by
one ulp, which size the tolerances of tests/test_long_runs.py.  The
intersection-law compression stops at its first step in the reference
(spurious contacts on the overlap-free packing); its fixture holds that step.
Run from the repository root:

    python tests/golden/make_long_runs.py [c0] [c1]
"""
import math
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from xdem_b200 import abi, inputs  # noqa: E402
from xdem_b200.world import make_control, make_params  # noqa: E402

C0_N = 1024
C0_STEPS = 10_000
C0_SAMPLE = 500
C1_N = 512
C1_RATE = -1e-4
C1_STOP = 1e-3 * inputs.KN


def strain_compress(world_cls, p, box, dt, phi_target, steps, relax, damping=0.1, method=0):
    """Strain-controlled compression of `p` to phi_target in about `steps`
    steps, then `relax` steps at the final box, by the given CPU world
    (the reference's own laws); returns the particle dict and the box."""
    prm = make_params(abi.WORLD_PERIODIC_CONTROL, dt, box, inputs.KN, inputs.KT,
                      inputs.RESTITUTION, inputs.FRICTION, global_damping=damping,
                      ellipse_method=method)
    w = world_cls(prm)
    w.set_particles(p)
    vol = float(p["volume"].sum())
    phi0 = vol / ((box[1] - box[0]) * (box[3] - box[2]))
    s_step = math.sqrt(phi0 / phi_target) ** (1.0 / steps)
    ctl = make_control(box_law=abi.BOX_STRAIN, reset_rattlers=False)
    done = 0
    while done < 3 * steps:
        b = w.getBoundary()
        L = b[1] - b[0]
        s_rem = math.sqrt(vol / (L * (b[3] - b[2])) / phi_target)
        if s_rem >= 1.0 - 1e-12:
            break
        left = max(1, int(math.ceil(math.log(s_rem) / math.log(s_step))))
        chunk = min(200, left)
        per = s_rem ** (1.0 / chunk) if chunk == left else s_step
        ctl.p0 = ctl.p1 = (per - 1.0) / (L * dt)
        w.run(chunk, ctl)
        done += chunk
    if relax:
        w.run(relax, make_control())
    st = w.get_state()
    q = dict(p)
    for k in ("x", "y", "vx", "vy", "rot", "rot_vel"):
        q[k] = st[k].copy()
    return q, np.array(w.getBoundary())


def c0_inputs(seed=2026):
    p, box = inputs.disc_system(C0_N, phi_rsa=0.50, phi=None, seed=seed, vel_sigma=0.01)
    dt = inputs.time_step(p)
    q, box = strain_compress(oracle.RefWorld, p, box, dt, 0.70, steps=3000, relax=1000)
    rng = np.random.default_rng(seed + 5)
    q["vx"] = rng.normal(0.0, 0.01, C0_N)
    q["vy"] = rng.normal(0.0, 0.01, C0_N)
    q["rot_vel"] = np.zeros(C0_N)
    q["is_rattler"] = np.zeros(C0_N, np.int32)
    return q, box, dt


def run_c0(world_cls, p, box, dt):
    prm = make_params(abi.WORLD_PERIODIC, dt, box, inputs.KN, inputs.KT, inputs.RESTITUTION,
                      inputs.FRICTION)
    w = world_cls(prm)
    w.set_particles(p)
    ctl = make_control(update_stress=True)
    stress, ncont, ke = [], [], []
    for _ in range(C0_STEPS // C0_SAMPLE):
        w.run(C0_SAMPLE, ctl)
        stress.append(w.getStress())
        ncont.append(w.count_contacts())
        ke.append(w.getKineticEnergy())
    return {"stress": np.array(stress), "contacts": np.array(ncont), "ke": np.array(ke),
            "state": w.get_state(), "contact_list": w.get_contacts(), "z_phi": w.quadron_z_phi()}


def perturbed(p, k):
    q = dict(p)
    q["vx"] = p["vx"].copy()
    q["vx"][k % len(q["vx"])] = np.nextafter(q["vx"][k % len(q["vx"])], 1.0)
    return q


def make_c0():
    t = time.time()
    p, box, dt = c0_inputs()
    phi = float(p["volume"].sum()) / ((box[1] - box[0]) * (box[3] - box[2]))
    print(f"c0 packing phi {phi:.4f} in {time.time() - t:.1f}s", flush=True)
    ref = run_c0(oracle.RefWorld, p, box, dt)
    print(f"c0 reference done {time.time() - t:.1f}s, contacts {ref['contacts'][-1]}, "
          f"z_phi {ref['z_phi']}", flush=True)
    port = run_c0(oracle.PortWorld, p, box, dt)
    spread = [run_c0(oracle.RefWorld, perturbed(p, 37 * k + 1), box, dt) for k in range(3)]
    arrs = {f"p_{k}": v for k, v in p.items() if isinstance(v, np.ndarray)}
    arrs["box"] = box
    arrs["dt"] = np.array(dt)
    arrs["sample_every"] = np.array(C0_SAMPLE)
    for tag, r in (("ref", ref), ("port", port)):
        arrs[f"{tag}_stress"] = r["stress"]
        arrs[f"{tag}_contacts"] = r["contacts"]
        arrs[f"{tag}_ke"] = r["ke"]
        arrs[f"{tag}_z_phi"] = r["z_phi"]
        for k, v in r["state"].items():
            arrs[f"{tag}_s_{k}"] = v
    for k in ("id_i", "id_j", "fn_x", "fn_y", "ft_x", "ft_y"):
        arrs[f"ref_c_{k}"] = ref["contact_list"][k]
    arrs["spread_stress"] = np.array([r["stress"] for r in spread])
    arrs["spread_z_phi"] = np.array([r["z_phi"] for r in spread])
    arrs["spread_x"] = np.array([r["state"]["x"] for r in spread])
    np.savez_compressed(os.path.join(HERE, "long_c0_discs.npz"), **arrs)
    d_port = np.max(np.abs(port["stress"] - ref["stress"])) / np.max(np.abs(ref["stress"]))
    d_spread = max(np.max(np.abs(r["stress"] - ref["stress"])) for r in spread) / np.max(
        np.abs(ref["stress"]))
    print(f"c0 written {time.time() - t:.1f}s; stress: port-ref {d_port:.3e}, "
          f"1-ulp spread {d_spread:.3e}; z_phi port {port['z_phi']} ref {ref['z_phi']}")


def ellipse_rsa(n, phi, seed, max_tries=2_000_000):
    """Random sequential addition of ellipses (b ~ U[0.4, 0.6], a = 1.5 b,
    orientations U[0, pi)) into a square box at solid fraction phi, largest
    first, with no two ellipses in contact by the compiled reference's own
    closest-approach test (calculateContactGeometry)."""
    rng = np.random.default_rng(seed)
    b = inputs.c1_b(rng, n)
    asp = inputs.c1_aspect(rng, n)
    a = asp * b
    rot = rng.uniform(0.0, np.pi, n)
    box = inputs.box_for(float(np.sum(np.pi * a * b)), phi)
    L = box[1] - box[0]
    order = np.argsort(-a, kind="stable")
    xs = np.zeros(n)
    ys = np.zeros(n)
    placed = []
    amax = float(a.max())
    tries = 0
    for i in order:
        while True:
            tries += 1
            if tries > max_tries:
                raise RuntimeError("ellipse RSA did not reach the solid fraction")
            x, y = rng.uniform(box[0], box[1]), rng.uniform(box[2], box[3])
            if placed:
                P = np.array(placed)
                dx = xs[P] - x
                dy = ys[P] - y
                dx -= L * np.round(dx / L)
                dy -= L * np.round(dy / L)
                near = np.nonzero(dx * dx + dy * dy < (a[i] + a[P]) ** 2)[0]
                if len(near):
                    k = P[near]
                    m = len(k)
                    pi = np.stack([np.ones(m), np.full(m, a[i]), np.full(m, asp[i]), np.full(m, x),
                                   np.full(m, y), np.zeros(m), np.zeros(m), np.full(m, rot[i]),
                                   np.zeros(m)], 1)
                    pj = np.stack([np.ones(m), a[k], asp[k], x + dx[near], y + dy[near],
                                   np.zeros(m), np.zeros(m), rot[k], np.zeros(m)], 1)
                    out, _ = oracle.pair_geometry(pi, pj, np.zeros((m, 4)),
                                                  abi.ELLIPSE_CLOSEST_APPROACH, "ref")
                    if out[:, 0].any():
                        continue
            xs[i], ys[i] = x, y
            placed.append(i)
            break
    zero = np.zeros(n)
    p = inputs.assemble(np.ones(n, np.int32), a, asp, xs, ys, zero, zero, rot, zero)
    return p, box, tries


C1_SAMPLE = 20_000
C1_MAX_STEPS = 2_000_000


def run_c1(world_cls, p, box, dt, method, max_steps=C1_MAX_STEPS, stop=True):
    """The compression of long_c1: strain control at C1_RATE with the stress
    updated every step, until trace(stress)/2 >= C1_STOP (or max_steps);
    samples every C1_SAMPLE steps."""
    prm = make_params(abi.WORLD_PERIODIC_CONTROL, dt, box, inputs.KN, inputs.KT,
                      inputs.RESTITUTION, inputs.FRICTION, ellipse_method=method)
    w = world_cls(prm)
    w.raise_mask = ~abi.ERR_NEWTON
    w.set_particles(p)
    ctl = make_control(update_stress=True, box_law=abi.BOX_STRAIN, p0=C1_RATE, p1=C1_RATE,
                       stop_pressure=C1_STOP if stop else None)
    steps, stress, phis = 0, [], []
    vol = float(p["volume"].sum())
    while steps < max_steps:
        done = w.run(min(C1_SAMPLE, max_steps - steps), ctl)
        steps += done
        b = w.getBoundary()
        stress.append(w.getStress())
        phis.append(vol / ((b[1] - b[0]) * (b[3] - b[2])))
        print(f"  {world_cls.__name__} step {steps}: phi {phis[-1]:.5f}, "
              f"p {(stress[-1][0] + stress[-1][3]) / 2:.4g}", flush=True)
        if done < C1_SAMPLE:
            break
    b = np.array(w.getBoundary())
    return {"steps": steps, "box": b, "phi": vol / ((b[1] - b[0]) * (b[3] - b[2])),
            "stress": np.array(stress), "phis": np.array(phis), "z_phi": w.quadron_z_phi(),
            "contacts": w.count_contacts(), "state": w.get_state()}


# The compiled reference's closest-approach compression stops returning
# between steps 10,000 and 20,000 of this run (its Newton loop,
# EllipticParticle.cpp:621, has no cap); it is pinned against the restatement
# on the first C1_REF_PREFIX steps, and the restatement runs the rest.
C1_REF_PREFIX = 10_000


def make_c1(method, tag, seed=7):
    t = time.time()
    p, box, tries = ellipse_rsa(C1_N, 0.50, seed)
    dt = inputs.time_step(p)
    print(f"c1 {tag}: rsa {tries} tries, {time.time() - t:.1f}s", flush=True)
    arrs = {f"p_{k}": v for k, v in p.items() if isinstance(v, np.ndarray)}
    arrs["box0"] = box
    arrs["dt"] = np.array(dt)
    arrs["method"] = np.array(method)
    arrs["rate"] = np.array(C1_RATE)
    arrs["stop_pressure"] = np.array(C1_STOP)
    arrs["sample_every"] = np.array(C1_SAMPLE)
    if method == abi.ELLIPSE_CLOSEST_APPROACH:
        ref = run_c1(oracle.RefWorld, p, box, dt, method, max_steps=C1_REF_PREFIX, stop=False)
        pre = run_c1(oracle.PortWorld, p, box, dt, method, max_steps=C1_REF_PREFIX, stop=False)
        arrs["prefix_steps"] = np.array(C1_REF_PREFIX)
        for name, r in (("ref_prefix", ref), ("port_prefix", pre)):
            for k in ("x", "y", "vx", "vy", "rot", "rot_vel"):
                arrs[f"{name}_s_{k}"] = r["state"][k]
            arrs[f"{name}_stress"] = r["stress"][-1]
            arrs[f"{name}_contacts"] = np.array(r["contacts"])
        d = max(np.max(np.abs(ref["state"][k] - pre["state"][k])) / np.max(np.abs(ref["state"][k]))
                for k in ("x", "y", "vx", "vy", "rot"))
        print(f"c1 {tag}: prefix of {C1_REF_PREFIX} steps, restatement vs reference state {d:.3e}, "
              f"contacts {pre['contacts']} {ref['contacts']}", flush=True)
        full = run_c1(oracle.PortWorld, p, box, dt, method)
        source = "C restatement (the compiled reference does not return on this run)"
    else:
        full = run_c1(oracle.RefWorld, p, box, dt, method)
        source = "compiled reference"
    print(f"c1 {tag}: {source}: {full['steps']} steps, phi {full['phi']:.5f}, "
          f"z_phi {full['z_phi']}, {time.time() - t:.0f}s", flush=True)
    arrs["source"] = np.array(source)
    for k in ("steps", "box", "phi", "stress", "phis", "z_phi", "contacts"):
        arrs[f"full_{k}"] = np.asarray(full[k])
    if full["steps"] > 1:
        spread = []
        for k in range(2):
            q = dict(p)
            q["rot"] = p["rot"].copy()
            q["rot"][53 * k + 2] = np.nextafter(q["rot"][53 * k + 2], 10.0)
            spread.append(run_c1(oracle.PortWorld, q, box, dt, method))
            print(f"c1 {tag}: 1-ulp run {k}: {spread[-1]['steps']} steps, phi "
                  f"{spread[-1]['phi']:.5f}, z_phi {spread[-1]['z_phi']}", flush=True)
        for k in ("steps", "phi", "z_phi", "contacts"):
            arrs[f"spread_{k}"] = np.array([np.asarray(r[k]) for r in spread])
    else:
        for k in ("x", "y", "vx", "vy", "rot", "rot_vel"):
            arrs[f"full_s_{k}"] = full["state"][k]
    np.savez_compressed(os.path.join(HERE, f"long_c1_{tag}.npz"), **arrs)
    print(f"c1 {tag} written, {time.time() - t:.0f}s", flush=True)


def main():
    if not oracle.ref_available():
        sys.exit("the compiled reference (oracle/_ref) is required")
    which = set(sys.argv[1:]) or {"c0", "c1"}
    if "c0" in which:
        make_c0()
    if "c1" in which:
        make_c1(abi.ELLIPSE_CLOSEST_APPROACH, "closest")
        make_c1(abi.ELLIPSE_INTERSECTION, "intersection")


if __name__ == "__main__":
    main()
