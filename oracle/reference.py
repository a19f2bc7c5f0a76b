"""REFERENCE BUILD (test infrastructure) -- runs oracle/_ref/ref_run, the reference MaBoSS.GPU
trajectory path compiled from its own sources by oracle/refbuild/Makefile, and reads its output.

Only tests/ and bench.py's reference arm use this module; the engine never does. ref_run runs on
the GPU (the reference is CUDA code); it refuses, before any GPU work, inputs for which the
reference's own index arithmetic would leave its buffers (exit code 3, see harness.cu).
"""
from __future__ import annotations

import json
import os
import subprocess
import tempfile

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_RUN = os.path.join(_HERE, "_ref", "ref_run")


class Refused(RuntimeError):
    """ref_run declined the input (the reference's int sizes or window indices would overflow)."""


def available() -> bool:
    return os.path.exists(REF_RUN)


def read_dump(path: str) -> dict:
    """The raw statistics of the reference's plugins (harness.cu: write_dump)."""
    with open(path, "rb") as f:
        buf = f.read()
    if buf[:8] != b"MBREF001":
        raise ValueError("not a ref_run dump")
    n, nodes, words, ni, T, S, disc, trans, nfix = (int(x) for x in np.frombuffer(buf, np.int64, 9, 8))
    max_time, tick = np.frombuffer(buf, np.float32, 2, 8 + 72)
    off = 8 + 72 + 8

    def take(dtype, count):
        nonlocal off
        a = np.frombuffer(buf, dtype, count, off).copy()
        off += a.nbytes
        return a

    disc = bool(disc)
    win = take(np.int32 if disc else np.float32, T * S).reshape(T, S)
    h = take(np.float32, T)
    final = take(np.int32, S)
    fstates = take(np.uint32, nfix * words).reshape(nfix, words)
    fcounts = take(np.int32, nfix)
    n32 = np.float32(n)
    tick32 = np.float32(tick)
    if disc:
        # window_average_small.cpp:126-131: (float)occurences / (float)n_trajectories
        probs = win.astype(np.float32) / n32
        th = h / n32
    else:
        # window_average_small.cpp:133-137: cumul_slices / (n_trajectories * window_size)
        probs = win / np.float32(n32 * tick32)
        th = (h / n32) / tick32
    return dict(n=n, nodes=nodes, state_words=words, noninternal=ni, windows=T, bins=S, discrete=disc,
                transitions=trans, max_time=float(max_time), time_tick=float(tick), window=win,
                probs=probs.astype(np.float64), th=th.astype(np.float64), final=final, fixed_states=fstates,
                fixed_counts=fcounts)


def run(bnd_path: str, cfg_path: str, samples: int | None = None, seed: int | None = None, warmup: int = 0,
        runs: int = 1, dump: bool = True, csv_prefix: str | None = None, timeout: float = 3600) -> dict:
    """Run the reference build once (plus warm-up and timed runs); returns the JSON summary
    (transitions, compile_s, device_ms and host_ms per timed run) and, with `dump`, the raw
    statistics of the last run under "result"."""
    if not available():
        raise FileNotFoundError(REF_RUN + " is not built (make -C oracle/refbuild)")
    with tempfile.TemporaryDirectory() as tmp:
        cmd = [REF_RUN, "--warmup", str(warmup), "--runs", str(runs)]
        if samples is not None:
            cmd += ["--samples", str(int(samples))]
        if seed is not None:
            cmd += ["--seed", str(int(seed))]
        dump_path = os.path.join(tmp, "dump.bin")
        if dump:
            cmd += ["--dump", dump_path]
        if csv_prefix:
            cmd += ["--csv", csv_prefix]
        cmd += [bnd_path, cfg_path]
        p = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
        lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
        summary = json.loads(lines[-1]) if lines else {}
        if p.returncode == 3:
            raise Refused(summary.get("refused", p.stderr.strip()))
        if p.returncode != 0:
            raise RuntimeError(f"ref_run failed ({p.returncode}): {p.stderr.strip()[-2000:]} {p.stdout[-2000:]}")
        if dump:
            summary["result"] = read_dump(dump_path)
        return summary


def run_text(bnd_text: str, cfg_text: str, **kw) -> dict:
    """run() on model text (written to a temporary .bnd/.cfg pair)."""
    with tempfile.TemporaryDirectory() as tmp:
        b, c = os.path.join(tmp, "m.bnd"), os.path.join(tmp, "m.cfg")
        with open(b, "w") as f:
            f.write(bnd_text)
        with open(c, "w") as f:
            f.write(cfg_text)
        return run(b, c, **kw)
