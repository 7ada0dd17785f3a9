"""Generate the golden fixtures of tests/golden from the reference's own
kernel bodies (oracle/_ref/libref.so, built from the reference checkout by
oracle/Makefile).  Run from the repository root:

    python tests/golden/make_golden.py

Each case stores the seeded input scene as a reference binary (<name>.bin)
and the reference state after `steps` time steps (<name>.npz).  The fixtures
travel with the tree, so the GPU tests can check against them without the
reference checkout.
"""
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))

import pyoracle  # noqa: E402
from sphere_b200 import scenes  # noqa: E402
from sphere_b200.spherebin import Spherebin  # noqa: E402
from sphere_b200.state import config_from_spherebin, state_from_spherebin  # noqa: E402


def io_scene():
    # tests/io_tests.py:8-15: 100 particles, no gravity, no overlap
    sb = Spherebin(np_=100, nw=1, sid="io_null_step")
    rng = np.random.default_rng(7)
    sb.generateRadii(rng=rng)
    sb.defaultParams()
    sb.initRandomGridPos(g=np.zeros(3), rng=rng)
    sb.initTemporal(current=0.0, total=0.0)
    sb.time_total = 2.0 * sb.time_dt
    sb.time_file_dt = sb.time_dt
    return sb


CASES = [
    ("box_256", lambda: scenes.collision(n=256, seed=101, periodic=0, sid="box_256"), 30),
    ("periodic_256", lambda: scenes.collision(n=256, seed=102, periodic=1, sid="periodic_256"), 30),
    ("periodic_x_wall_256", lambda: scenes.collision(n=256, seed=103, periodic=2, nw=1,
                                                       sid="periodic_x_wall_256"), 30),
    ("bonded_32", lambda: scenes.bonded(nx=2, ny=2, nz=2, sigma_b=1e30, tau_b=1e30, sid="bonded_32"), 30),
    ("io_null_step", io_scene, 3),
]

FIELDS = ("x", "vel", "angvel", "angpos", "xysum", "es", "ev", "force", "torque", "es_dot",
          "ev_dot", "p", "contacts", "walls_nx", "walls_mvfd", "walls_vel0", "bonds",
          "bonds_delta", "bonds_omega")


def main():
    pyoracle.build(ref=True)
    lib = pyoracle.load("ref")
    index = {"generator": "tests/golden/make_golden.py", "oracle": "oracle/_ref (reference kernels)",
             "cases": []}
    for name, make, steps in CASES:
        sb = make()
        sb.sid = name
        sb.writebin(path=HERE / f"{name}.bin", verbose=False)
        cfg = config_from_spherebin(sb)
        st = state_from_spherebin(sb)
        run = pyoracle.OracleRun(lib, cfg, st)
        rc = run.step(steps, 1)
        if rc != 0:
            raise SystemExit(f"{name}: reference harness returned {rc}")
        out = {f: np.asarray(getattr(st, f)) for f in FIELDS}
        out["perm"] = run.perm.copy()
        out["delta_t_active"] = st.delta_t[st.contacts != sb.np]
        np.savez_compressed(HERE / f"{name}.npz", **out)
        index["cases"].append({"name": name, "input": f"{name}.bin", "expected": f"{name}.npz",
                               "steps": steps, "np": int(sb.np),
                               "active_contacts": int((st.contacts != sb.np).sum())})
        print(name, "active contacts", index["cases"][-1]["active_contacts"])
    (HERE / "index.json").write_text(json.dumps(index, indent=1) + "\n")


if __name__ == "__main__":
    main()
