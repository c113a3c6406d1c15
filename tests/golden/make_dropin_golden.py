"""Golden outputs of drivers built on the CPU from the reference sources with the Eigen-API shim,
for the comparison with the same drivers linked against the drop-in library (tests/test_gpu_dropin.py).

* dropin_oscillations/: the reference's own oscillations driver (oscillations.cpp, unchanged,
  oracle/_ref/refdrv/oscillations).  Input: the icosphere nu = 10 written by tests/plyio.py as
  ../python_utils/icosphere/ico-10.ply (the path the driver opens); arguments radius 3e-6 m, acoustic
  pressure 5e4 Pa.  The driver's first three exports (mesh-0..mesh-2) are copied.
* dropin_check/: oracle/dropin_check.cpp (oracle/_ref/refdrv/dropin_check) on the icosphere nu = 7:
  its three exports ref-0..ref-2 and its exterior-potential probe (ref_exterior.txt).  This driver is
  reproducible bit for bit across thread counts.
* pinned_check/: oracle/pinned_check.cpp (oracle/_ref/refdrv/pinned_check, the reference's ColocSimPin)
  on the wall cap nu = 6 (bem_b200.mesh.wall_cap): its three exports ref-0..ref-2 and its printed
  block and pinned-vertex lines (ref_stdout.txt).  The reference's ColocSimPin assembly adds the
  triangles' columns in thread order (omp_set_num_threads(num_threads), 100 by default), so two runs
  differ by rounding (6e-16 relative in these lines).

Run from the repository root after `make -C oracle refdrivers`; takes a few minutes
(`--only pinned` for the last part alone).
"""
import argparse
import os
import shutil
import subprocess
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "bem-bubbles_b200"))
sys.path.insert(0, os.path.dirname(HERE))
from bem_b200 import mesh  # noqa: E402
from plyio import write_ply  # noqa: E402

ARGS = ["3e-6", "50000", "out"]
EXPORTS = 3


def pinned_check():
    out_dir = os.path.join(HERE, "pinned_check")
    os.makedirs(out_dir, exist_ok=True)
    with tempfile.TemporaryDirectory() as tmp:
        v, f = mesh.wall_cap(6)
        write_ply(os.path.join(tmp, "cap-6.ply"), v, f)
        os.makedirs(os.path.join(tmp, "borderprojects"))
        exe = os.path.join(ROOT, "oracle", "_ref", "refdrv", "pinned_check")
        r = subprocess.run([exe, os.path.join(tmp, "cap-6.ply"), os.path.join(out_dir, "ref")], check=True,
                           capture_output=True, text=True, cwd=tmp)
        with open(os.path.join(out_dir, "ref_stdout.txt"), "w") as fh:
            fh.writelines(ln + "\n" for ln in r.stdout.splitlines() if ln.startswith(("block ", "pinned ")))
    print("wrote", out_dir)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", choices=["pinned"], default=None)
    if ap.parse_args().only == "pinned":
        pinned_check()
        return
    exe = os.path.join(ROOT, "oracle", "_ref", "refdrv", "oscillations")
    out_dir = os.path.join(HERE, "dropin_oscillations")
    os.makedirs(out_dir, exist_ok=True)
    with tempfile.TemporaryDirectory() as tmp:
        os.makedirs(os.path.join(tmp, "python_utils", "icosphere"))
        run = os.path.join(tmp, "run")
        os.makedirs(os.path.join(run, "out"))
        v, f = mesh.icosphere(10)
        write_ply(os.path.join(tmp, "python_utils", "icosphere", "ico-10.ply"), v, f)
        proc = subprocess.Popen([exe] + ARGS, cwd=run, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        want = os.path.join(run, "out", f"mesh-{EXPORTS}.ply")  # written once mesh-{EXPORTS-1} is final
        while not os.path.exists(want) and proc.poll() is None:
            time.sleep(1.0)
        time.sleep(1.0)
        proc.kill()
        proc.wait()
        for k in range(EXPORTS):
            shutil.copy(os.path.join(run, "out", f"mesh-{k}.ply"), os.path.join(out_dir, f"mesh-{k}.ply"))
    print("wrote", out_dir)
    check_dir = os.path.join(HERE, "dropin_check")
    os.makedirs(check_dir, exist_ok=True)
    with tempfile.TemporaryDirectory() as tmp:
        v, f = mesh.icosphere(7)
        write_ply(os.path.join(tmp, "ico-7.ply"), v, f)
        exe = os.path.join(ROOT, "oracle", "_ref", "refdrv", "dropin_check")
        r = subprocess.run([exe, os.path.join(tmp, "ico-7.ply"), os.path.join(check_dir, "ref")], check=True,
                           capture_output=True, text=True)
        with open(os.path.join(check_dir, "ref_exterior.txt"), "w") as fh:
            fh.writelines(ln + "\n" for ln in r.stdout.splitlines() if ln.startswith("exterior "))
    print("wrote", check_dir)
    pinned_check()


if __name__ == "__main__":
    main()
