"""Generate tests/golden/mpmath_checks.json: the oracle's .fds renders of a few views,
each checked here by the reference's own independent mpmath checker (tools/oracle.py of
junovhs/fractodactyl: direct iteration z <- z^2 + c at depth + 128 bits, no perturbation,
class / nu / de / normal gated as output-pixel displacements), recorded with the FNV-1a
hash of the checked bytes and the checker's verdict. The tests re-render each view and
compare hashes, so the bytes mpmath passed stay the oracle's and (through the product's
byte-equality tests) the route's.

Runs only where the reference tree is present (the checker is not copied here).
usage: python tests/golden/make_mpmath_checks.py REFERENCE_ROOT
"""
import json
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(HERE)), "oracle"))

import fdref  # noqa: E402

# (name, re, im, width, nx, ny, max_iter, rotation, BLA eps or None)
VIEWS = [
    ("f64-rotated", "-0.7453", "0.1127", "0.0065", 64, 36, 4_000, 0.3, None),
    ("f64-period3-bulb", "-0.1226", "0.7449", "0.3", 48, 32, 2_000, 0.0, None),
    ("f64-main-components", "-0.75", "0.1", "0.4", 48, 32, 2_000, 0.0, None),
    ("fixed-seahorse", "-0.7436438870371587", "0.1318259042053120", "1e-12", 64, 36, 20_000, 0.0, None),
    ("fixed-seahorse-bla", "-0.7436438870371587", "0.1318259042053120", "1e-12", 64, 36, 20_000, 0.0, 2.0 ** -50),
    ("scaled-1e-300", "0", "1", "1e-300", 64, 36, 5_000, 0.0, None),
    ("scaled-1e-300-bla", "0", "1", "1e-300", 64, 36, 5_000, 0.0, 2.0 ** -50),
]
K = 6


def render(v):
    name, re_, im_, width, nx, ny, it, rot, eps = v
    job = fdref.make_job(re_, im_, width, nx, ny, it, rotation=rot,
                         columns=fdref.COL_NU | fdref.COL_DE | fdref.COL_NORMAL, threads=4)
    ref = bla = None
    if eps is not None:
        ref = fdref.Ref.for_job(job)
        dc, e = fdref.bla_dc_bound(job)
        bla = fdref.Bla(ref, eps, dc, e)
    return fdref.render_fds(job, ref, bla)


def main(root):
    checker = os.path.join(root, "tools", "oracle.py")
    out = []
    with tempfile.TemporaryDirectory() as tmp:
        for v in VIEWS:
            data = render(v)
            path = os.path.join(tmp, v[0] + ".fds")
            with open(path, "wb") as f:
                f.write(data)
            r = subprocess.run([sys.executable, checker, path, "--k", str(K)], capture_output=True, text=True,
                               timeout=1800)
            stats = json.loads(r.stdout)
            keep = {k: stats[k] for k in ("kernel", "samples", "escaped", "class_mismatch", "nu_px_err", "de_px_err",
                                          "normal_px_err", "bits", "ok")}
            out.append({"name": v[0], "re": v[1], "im": v[2], "width": v[3], "nx": v[4], "ny": v[5],
                        "max_iter": v[6], "rotation": v[7], "bla_eps": v[8], "k": K,
                        "fnv": "0x%016x" % fdref.fnv1a64(data), "checker": keep, "exit": r.returncode})
            print(v[0], keep)
    with open(os.path.join(HERE, "mpmath_checks.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {sys.argv[0]} REFERENCE_CHECKOUT (the junovhs/fractodactyl source tree)")
    main(sys.argv[1])
