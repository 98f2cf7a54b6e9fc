"""Dense packings made on the GPU: strain-controlled compression of an RSA
packing in a PeriodicControlWorld (updatePeriodicBoundary_strainControl,
PeriodicControlWorld.cpp:124-135), then relaxation at the final box, as the
reference's compression drivers do (mainIsoCircPack_WCCM.cpp:46-126).
"""
import math

import numpy as np

from . import abi, inputs
from .world import World, make_control, make_params


def compress(p, box, phi_target, dt, steps=4000, relax=2000, global_damping=0.1,
             ellipse_method=abi.ELLIPSE_CLOSEST_APPROACH, max_contacts=0):
    """Compresses the particles `p` (dict of inputs.assemble) in `box` to solid
    fraction `phi_target` in about `steps` steps of strain control, then runs
    `relax` steps at the final box.  Returns (particles, contacts, box, info);
    the particle dict is a copy with the new dynamic state."""
    prm = make_params(abi.WORLD_PERIODIC_CONTROL, dt, box, inputs.KN, inputs.KT,
                      inputs.RESTITUTION, inputs.FRICTION, global_damping=global_damping,
                      ellipse_method=ellipse_method, max_contacts=max_contacts)
    w = World(prm)
    # a fast compression sends a few deeply overlapping pairs into the
    # closest-approach Newton cycle; the capped solver reports it and goes on
    w.raise_mask = ~abi.ERR_NEWTON
    w.set_particles(p)
    vol = float(p["volume"].sum())
    area0 = (box[1] - box[0]) * (box[3] - box[2])
    phi0 = vol / area0
    # strain control scales the box by s = 1 + r*L*dt per step; the rate is
    # set chunk by chunk so that the compression reaches phi_target from below
    s_step = math.sqrt(phi0 / phi_target) ** (1.0 / steps)
    ctl = make_control(box_law=abi.BOX_STRAIN, reset_rattlers=False)
    done = 0
    while done < 3 * steps:
        b = w.getBoundary()
        L = b[1] - b[0]
        phi = vol / (L * (b[3] - b[2]))
        s_rem = math.sqrt(phi / phi_target)  # < 1 while below the target
        if s_rem >= 1.0 - 1e-7:
            break
        left = max(1, int(math.ceil(math.log(s_rem) / math.log(s_step))))
        chunk = min(200, left)
        per = s_rem ** (1.0 / chunk) if chunk == left else s_step
        ctl.p0 = ctl.p1 = (per - 1.0) / (L * dt)
        w.run(chunk, ctl)
        done += chunk
    b = w.getBoundary()
    phi = vol / ((b[1] - b[0]) * (b[3] - b[2]))
    if relax:
        w.run(relax, make_control())
    capped = w.newton_stats()[2]
    st = w.get_state()
    contacts = w.get_contacts()
    b = np.array(w.getBoundary())
    q = dict(p)
    for k in ("x", "y", "vx", "vy", "rot", "rot_vel"):
        q[k] = st[k].copy()
    q["is_rattler"] = st["is_rattler"].copy()
    w.close()
    return q, contacts, b, {"phi0": phi0, "phi": phi, "steps": done, "relax": relax,
                            "capped_newton": capped}
