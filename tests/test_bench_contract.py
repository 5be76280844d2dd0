"""bench.py's output contract on the CPU: the reference arm (the CPU kernel timed on a
bounded sample of the workload's rows) prints one JSON line with every key the bench
line carries, its cpu_baseline and e2e describing that same run; under a multi-rank
launch only rank 0 prints; and the CUDA arm, given no device, fails with a non-zero exit
and no bench line instead of falling back to the CPU."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BENCH = os.path.join(ROOT, "bench.py")


def _run(args, env=None, timeout=300):
    e = dict(os.environ)
    e.update(env or {})
    return subprocess.run([sys.executable, BENCH, *args], cwd=ROOT, env=e, capture_output=True, text=True,
                          timeout=timeout)


def test_reference_arm_line():
    r = _run(["--impl", "reference", "--config", "1", "--steps", "2", "--warmup", "3", "--cpu-seconds", "0.5"])
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    sys.path.insert(0, ROOT)
    import bench
    assert line["metric"] == bench.METRIC and line["unit"] == bench.UNIT
    assert line["impl"] == "reference"
    assert line["value"] > 0 and line["ms_per_step"] > 0
    assert (line["n_gpus"], line["steps"], line["warmup"]) == (1, 2, 3)
    assert line["higher_is_better"] is True and line["scaling"] == "weak" and line["vs_baseline"] is None
    assert line["dtype"] == "f64" and line["data"].startswith("synthetic")
    cfg = line["config"]
    assert cfg["workload"].startswith("c1-") and (cfg["nx"], cfg["ny"], cfg["max_iter"]) == (480, 270, 20_000)
    assert 0 < cfg["sample_rows"] <= cfg["ny"]
    cb = line["cpu_baseline"]
    assert cb["value"] == line["value"] and cb["unit"] == line["unit"] and cb["kind"] in ("port", "reference")
    assert cb["cores"] >= 1 and cb["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_silent():
    r = _run(["--impl", "reference", "--config", "1", "--steps", "1", "--warmup", "3"],
             env={"RANK": "1", "LOCAL_RANK": "1", "WORLD_SIZE": "2"})
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""


def test_cuda_arm_fails_without_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    r = _run(["--config", "1", "--steps", "1", "--warmup", "3", "--no-cpu"])
    assert r.returncode != 0
    assert not [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert "NO_DEVICE" in r.stderr or "CUDA" in r.stderr


@pytest.mark.parametrize("config", [1, 2])
def test_reference_arm_frame_is_the_bench_frame(config):
    """The reference arm reads its frame with json alone; it is the frame the CUDA arm
    renders (fractodactyl_b200.locations), field for field."""
    sys.path.insert(0, ROOT)
    import argparse

    import bench
    from fractodactyl_b200 import locations
    for extra in ({}, dict(nx=64, ny=36, tier="scaled")):
        a = argparse.Namespace(config=config, seed=2, nx=extra.get("nx", 0), ny=extra.get("ny", 0),
                               tier=extra.get("tier"))
        w, f = bench.workload(a), bench.frame_for(a)
        assert (w.name, w.bla_eps, w.period) == (f.name, f.bla_eps, f.period)
        assert vars(w.view) == {k: getattr(f.view, k) for k in ("center_re", "center_im", "width", "rotation")}
        for k in ("nx", "ny", "max_iter", "escape_radius", "columns", "tier"):
            assert getattr(w.params, k) == getattr(f.params, k), k


def test_reference_arm_loads_no_repo_library():
    """The CPU arm of configuration 2 (whose centre the route's recipe computes) runs the
    oracle only: libfdcuda.so is never mapped into its process."""
    code = ("import sys, runpy; sys.argv = ['bench.py', '--impl', 'reference', '--config', '2', '--steps', '1', "
            "'--warmup', '3', '--cpu-seconds', '0.2'];\n"
            "runpy.run_path('bench.py', run_name='__main__')\n"
            "maps = open('/proc/self/maps').read()\n"
            "assert 'liboracle.so' in maps\n"
            "print('MAPPED_FDCUDA' if 'libfdcuda.so' in maps else 'CLEAN')\n")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip().splitlines()[-1] == "CLEAN"
    line = json.loads([ln for ln in r.stdout.splitlines() if ln.startswith("{")][0])
    assert line["impl"] == "reference" and line["config"]["workload"] == "c2-1920x1080-1e-100-seed2"


@pytest.mark.parametrize("width,tier", [("0.0065", None), ("1e-20", None), ("1e-300", "scaled")])
def test_bench_parity_helpers_on_oracle_frames(width, tier):
    """bench.py's checks on the CPU: sample_offset gives each sample's offset as the grid
    forms it (the oracle's per-sample iteration there equals its frame render), the
    parity summary of a frame against itself is exact and catches a planted count error,
    and the direct-iteration report finds no miss on a plain frame of a shallow view."""
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np

    import bench
    import fdref
    from fractodactyl_b200 import route
    re_, im_, nx, ny, it = "-0.7453", "0.1127", 24, 16, 3000
    view, p = route.View(re_, im_, width), route.Params(nx, ny, max_iter=it, tier=tier, columns=("nu",))
    plane, t = route._setup(view, p)
    job = fdref.make_job(re_, im_, width, nx, ny, it, columns=fdref.COL_NU, tier=t, threads=2)
    ref = fdref.Ref.for_job(job)
    want = fdref.render(job, ref, None, raw=True)
    kinds = {"escaped": 0, "interior": 1, "unresolved": 2}
    for k in range(0, nx * ny, 7):
        ar, ai, oe = bench.sample_offset(plane, t, nx, ny, k)
        o = fdref.iterate(ref, None, extended=t == 2, derivative=False, ar=ar, ai=ai, offset_exp=oe, max_iter=it,
                          r2=1e20, c=(plane.c_re + ar, plane.c_im + ai) if t == 0 else None)
        assert kinds[o["kind"]] == want["cls"][k] & 3, k
        if o["kind"] == "escaped":
            assert o["n"] == want["n"][k] and (o["zr"], o["zi"]) == tuple(want["z"][k]), k
    same = bench.parity_vs_oracle(want, want, exact=True)
    assert same["class_equal"] == same["count_equal"] == same["z_bit_equal"] == same["dz_bit_equal"] == 1.0
    bad = dict(want, n=want["n"].copy())
    esc = np.flatnonzero((want["cls"] & 3) == 0)
    bad["n"][esc[0]] += 1
    worse = bench.parity_vs_oracle(bad, want, exact=True)
    assert worse["count_equal"] == 1.0 - 1.0 / (nx * ny) and worse["within_one"] == 1.0
    if t != 2:  # direct iteration of a few escaping samples of the shallow views
        cases = []
        for k in esc[:6]:
            ar, ai, oe = bench.sample_offset(plane, t, nx, ny, int(k))
            cases.append((re_, im_, plane.bits + 64, it, 1e10, ar, ai, oe,
                          {"plain": (0, int(want["n"][k]), float(want["nu"][k]))}))
        rep = bench.precision_vs_direct(fdref, cases, ["plain"], 60.0, 2)
        assert rep["samples"] == 6 and rep["plain"]["off_by_more_than_one"] == 0.0
