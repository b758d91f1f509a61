"""AddressSanitizer pass over the reference's own code on this path -- TEST INFRASTRUCTURE.

    make -C oracle asan && python oracle/asan_check.py

Runs the golden scenes (every sensor kind, Mie / RGD / HG media, interfaces, time bins,
filters, MixtureLayers, the Absorption recorder, StatisticsSensors, estimator mode)
through the reference's unmodified sources built with AddressSanitizer (the `asan`
flavour of oracle/Makefile).  Errors are reported and execution continues
(-fsanitize-recover=address, halt_on_error=0).  Prints every distinct report: its kind,
the access, and the first frame in the reference's sources, with a count.

The Python interpreter is not instrumented, so the sanitizer runtime is preloaded
(LD_PRELOAD), and leak detection is off (the interpreter keeps its objects to exit).
"""
from __future__ import annotations

import collections
import json
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)

SCENE_SETS = ("golden_scenes", "statistics_scenes", "mixture_scenes", "absorption_scenes",
              "estimator_scenes")

_CHILD = r"""
import os, sys
sys.path.insert(0, {repo!r}); sys.path.insert(0, os.path.join({repo!r}, "luminis-mc_b200"))
from tests.golden import make_golden as G
from luminis_mc_b200 import workloads as W
from oracle import pyoracle as O
lm = O.reference_module("asan"); lm.set_log_level(lm.LogLevel.off)
for spec in getattr(G, {scene_set!r})():
    cfg, hs, keep = W.build(lm, spec, n_photons=min(int(spec["n_photons"]), {max_photons}),
                            n_threads=1)
    lm.run_simulation_parallel(cfg)
    print("ran", spec["name"], flush=True)
"""

_ERROR = re.compile(r"ERROR: AddressSanitizer: ([\w-]+)")
_ACCESS = re.compile(r"^(READ|WRITE) of size (\d+)", re.M)
_FRAME = re.compile(r"#\d+ 0x[0-9a-f]+ in (.+?) (\S*/src/\S+?):(\d+)")


def libasan() -> str:
    return subprocess.run(["gcc", "-print-file-name=libasan.so"], check=True, capture_output=True,
                          text=True).stdout.strip()


def run(scene_set: str, max_photons: int = 2000) -> tuple[list[str], str]:
    env = dict(os.environ, LD_PRELOAD=libasan(),
               ASAN_OPTIONS="halt_on_error=0:detect_leaks=0:allocator_may_return_null=1")
    code = _CHILD.format(repo=REPO, scene_set=scene_set, max_photons=max_photons)
    p = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True)
    ran = [ln.split()[1] for ln in p.stdout.splitlines() if ln.startswith("ran ")]
    if p.returncode != 0:
        raise RuntimeError(f"{scene_set}: exit {p.returncode}\n{p.stderr[-4000:]}")
    return ran, p.stderr


def reports(stderr: str):
    """(kind, access, function, file:line) of every report, at its first frame in the
    reference's sources."""
    out = []
    for block in stderr.split("=================================================================")[1:]:
        m = _ERROR.search(block)
        if not m:
            continue
        a = _ACCESS.search(block)
        f = _FRAME.search(block)
        where = (f.group(1), f"{f.group(2).split('/src/')[-1]}:{f.group(3)}") if f else ("?", "?")
        out.append((m.group(1), f"{a.group(1)} {a.group(2)}" if a else "?", *where))
    return out


def main():
    summary = collections.Counter()
    scenes = []
    for s in SCENE_SETS:
        ran, err = run(s)
        scenes += ran
        summary.update(reports(err))
    print(json.dumps({"scenes": scenes,
                      "reports": [{"kind": k, "access": a, "function": fn, "at": at, "count": n}
                                  for (k, a, fn, at), n in summary.most_common()]}, indent=1))


if __name__ == "__main__":
    main()
