"""bench.py's command line, without a GPU: the options the benchmark driver and the profiling
commands use are there, and a timed FP64 run outside --solves-only is refused before any device
work."""
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(*args):
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], capture_output=True, text=True,
                          timeout=300)


def test_help_lists_the_options():
    r = _run("--help")
    assert r.returncode == 0
    for opt in ("--gpus", "--steps", "--warmup", "--impl", "--workload", "--scan-method", "--scan-blocks",
                "--precision", "--solves-only", "--ref-budget-s", "--scan-energies"):
        assert opt in r.stdout, opt


def test_fp64_precision_needs_solves_only():
    r = _run("--precision", "fp64")
    assert r.returncode == 2 and "--solves-only" in r.stderr
    r = _run("--precision", "fp64", "--solves-only", "--workload", "scan")
    assert r.returncode == 2
