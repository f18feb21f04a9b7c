"""Records the reference planner's output on the reference scene, as the
fixture the drop-in test compares the B200 run with.

GPUPRM's own planner (PRMSolver<4>::process_mpi5) runs with GPUPRM's own
CPU checker through oracle/_ref/prm_dropin (built by oracle/Makefile from
the reference sources) on prm/config1 (taken from the config1 fixture and
written in the reference's config-directory format), seed 0, the
parameters of prm/src/main.cpp (num 32, nbuf 2048, dq 0.01, D = H = 1,
blocksize 256).  The fixture keeps the planner's counters, a SHA-256 of
every file store_results writes (prmsolver.cpp:2947-3055) — of
connection.bin only its first byte is defined (a bool written as an int),
so that byte is kept instead — and a SHA-256 of the sequence of checker
calls the planner made with their free/not-free verdicts (the harness's
--trace records, codes reduced to verdicts: the planner reads only
whether a code is 0).

    python tests/golden/make_prm_golden.py
"""
from __future__ import annotations

import hashlib
import json
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from gpuprm_b200 import scenes  # noqa: E402

BIN = os.path.join(ROOT, "oracle", "_ref", "prm_dropin")
ARGS = ["--seed", "0", "--num", "32", "--nbuf", "2048", "--dq", "0.01", "--distD", "1.0", "--distH", "1.0",
        "--blocksize", "256", "--maxsteps", "10000"]
FIXTURE = os.path.join(HERE, "prm_dropin_config1.json")


def digest_outputs(out_dir: str) -> dict:
    files = {}
    for base, _, names in os.walk(out_dir):
        for n in sorted(names):
            p = os.path.join(base, n)
            rel = os.path.relpath(p, out_dir)
            data = open(p, "rb").read()
            files[rel] = data[:1].hex() if rel == "connection.bin" else hashlib.sha256(data).hexdigest()
    return files


def verdict_digest(trace_path: str) -> tuple[str, int, int]:
    """SHA-256 over the trace's records with every code replaced by its
    verdict (0 free, 1 not free); also the numbers of vertex calls and of
    edges."""
    import struct
    import numpy as np
    b = open(trace_path, "rb").read()
    h = hashlib.sha256()
    i = nv = ne = 0
    while i < len(b):
        t = b[i:i + 1]
        i += 1
        if t == b"V":
            code = struct.unpack("i", b[i + 16:i + 20])[0]
            h.update(b"V" + b[i:i + 16] + bytes([code != 0]))
            i += 20
            nv += 1
        elif t == b"E":
            n = struct.unpack("i", b[i:i + 4])[0]
            rec = np.frombuffer(b[i + 4:i + 4 + 36 * n], np.uint8).reshape(n, 36)
            codes = rec[:, 32:].copy().view(np.int32).ravel()
            h.update(b"E" + b[i:i + 4] + rec[:, :32].tobytes() + (codes != 0).astype(np.uint8).tobytes())
            i += 4 + 36 * n
            ne += n
        else:
            raise ValueError(f"bad trace record at byte {i - 1}")
    return h.hexdigest(), nv, ne


def run_planner(checker: str, work: str, extra=()) -> tuple[dict, dict]:
    """Runs the planner once in `work` (a fresh directory) with a verdict
    trace; returns its JSON line (plus the trace digest) and the digests of
    its stored results."""
    from make_golden import scene_from_npz
    import numpy as np
    sc = scene_from_npz(np.load(os.path.join(HERE, "config1.npz")))
    cfg = scenes.write_config_dir(sc, os.path.join(work, "config1"))
    out = os.path.join(work, "prmoutput")   # store_results removes and recreates it
    trace = os.path.join(work, "verdicts.trace")
    r = subprocess.run([BIN, "--checker", checker, "--config", cfg, "--out", out, "--trace", trace] + ARGS +
                       list(extra), capture_output=True, text=True, timeout=900)
    if r.returncode != 0:
        raise RuntimeError(f"prm_dropin failed ({r.returncode}): {r.stderr[-2000:]}")
    line = json.loads(r.stdout.strip().splitlines()[-1])
    line["verdict_digest"], line["vertex_calls"], line["edges"] = verdict_digest(trace)
    return line, digest_outputs(out)


def main():
    with tempfile.TemporaryDirectory() as work:
        line, files = run_planner("ref", work)
    keep = {k: line[k] for k in ("num_nodes", "rand_nodes_all", "rand_nodes_accepted", "edge_step_checks",
                                 "start_free", "end_free", "verdict_digest", "vertex_calls", "edges")}
    json.dump({"args": ARGS, "counters": keep, "files": files, "reference_plan_seconds": line["plan_seconds"]},
              open(FIXTURE, "w"), indent=1, sort_keys=True)
    print("wrote", FIXTURE, keep)


if __name__ == "__main__":
    main()
