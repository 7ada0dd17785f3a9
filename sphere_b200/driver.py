"""Host time loop of ``DEM::startTime`` (``src/device.cu:576-1299``), in Python.

The reference advances ``time.current`` (double) by ``dt`` each step while
``time.current <= time.total``, and counts ``filetimeclock`` -- declared
``float`` (``src/device.cu:594``) -- up by ``dt`` to decide when to write the
next output file (``device.cu:1109-1188``).  ``schedule`` reproduces that
bookkeeping on the host so a run can be issued as a few long ``sph_step``
calls between output files instead of one call per step; ``run`` drives any
stepper (the GPU ``Simulation`` or a CPU oracle in tests) through it and
writes the reference's output files.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np


def schedule(time_current: float, time_total: float, dt: float, file_dt: float):
    """Steps of the reference loop that end in an output file.

    Returns (output_steps, total_steps, times) where output_steps lists the
    1-based step numbers after which an output is written and times the
    ``time.current`` value at each of those outputs."""
    t = float(time_current)
    ftc = np.float32(0.0)
    step = 0
    outs, times = [], []
    while t <= time_total:
        step += 1
        t = t + dt
        ftc = np.float32(np.float64(ftc) + dt)
        if np.float64(ftc) >= file_dt:
            outs.append(step)
            times.append(t)
            ftc = np.float32(0.0)
    return outs, step, times


def write_status(path: Path, current: float, total: float, step_count: int):
    """``output/<sid>.status.dat`` (``src/device.cu:656-662``)."""
    pct = 100.0 * current / total if total else 0.0
    path.write_text("%2.4e %2.4e %d\n" % (current, pct, step_count))


def run(sb, stepper, outdir="output", write_files=True):
    """Advance ``sb`` through its whole time interval with ``stepper``.

    ``stepper(nsteps)`` advances the device state; ``stepper.snapshot()``
    returns a Spherebin of the current state.  Files: output00000 with the
    input state, then one output per file interval, status.dat after each."""
    from .spherebin import Spherebin  # noqa: F401  (type of sb)
    out = Path(outdir)
    outs, total, times = schedule(sb.time_current, sb.time_total, sb.time_dt, sb.time_file_dt)
    if write_files:
        out.mkdir(parents=True, exist_ok=True)
        sb.writebin(path=out / f"{sb.sid}.output00000.bin", verbose=False)
        write_status(out / f"{sb.sid}.status.dat", sb.time_current, sb.time_total, sb.time_step_count)
    done = 0
    step_count = int(sb.time_step_count)
    last = sb
    for k, s in enumerate(outs):
        stepper(s - done)
        done = s
        step_count += 1
        last = stepper.snapshot()
        last.time_current = times[k]
        last.time_step_count = step_count
        if write_files:
            last.writebin(path=out / f"{sb.sid}.output{step_count:05d}.bin", verbose=False)
            write_status(out / f"{sb.sid}.status.dat", times[k], sb.time_total, step_count)
    if total > done:
        stepper(total - done)
    return last, outs, total
