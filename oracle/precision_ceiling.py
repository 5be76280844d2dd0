"""Accuracy ceiling of FP32-mantissa deltas, measured with the CPU oracle (test
infrastructure; no GPU, no product code).

The oracle's kernel is run twice over the same seeded subset of a view's samples: as the
reference's algorithm (binary64 deltas), and with every delta the kernel writes rounded
to `bits` mantissa bits, everything else (orbit, derivative, rebase test, bailout, BLA
radii, periodicity) left in binary64. At 24 bits that is an ideal FP32-mantissa delta:
no FP32 kernel can follow the binary64 deltas more closely, whatever its own shortcuts.
The escape-count agreement of the rounded runs with the binary64 run is the ceiling of
every FP32-delta form on that view. With --round-orbit the orbit point each plain step
multiplies the delta by is rounded too, as an FP32 recurrence holds its copy of Z.

    python oracle/precision_ceiling.py [--samples 20000] [--bits 24 32 40 48]

Views: configuration 2's seeded 1e-100 nucleus (1920x1080, 10^6 iterations, BLA from the
CPU builder, floatexp deltas), the 1e-12 seahorse view of configuration 1 (480x270,
2*10^4 iterations, bailout 2^8) and a 1e-28 view on the same spiral (256x144, 5*10^4).
Prints one JSON object per view and width.
"""
import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import fdref  # noqa: E402

EPS = 2.0 ** -50


def views():
    with open(os.path.join(HERE, "..", "fractodactyl_b200", "locations.json")) as f:
        c2 = [d for d in json.load(f)["c2"] if d["seed"] == 2][0]
    return [
        dict(name="c2-1920x1080-1e-100-seed2", re=c2["re"], im=c2["im"], width="1e-100", nx=1920, ny=1080,
             max_iter=1_000_000, escape_radius=1e10, tier="scaled", bla=EPS),
        dict(name="c1-480x270-1e-12", re="-0.7436438870371587", im="0.1318259042053120", width="1e-12", nx=480,
             ny=270, max_iter=20_000, escape_radius=256.0, tier=None, bla=None),
        dict(name="1e-28-256x144", re="-0.743643887037158704752191506114774",
             im="0.131825904205311970493132056385139", width="1e-28", nx=256, ny=144, max_iter=50_000,
             escape_radius=1e10, tier=None, bla=None),
    ]


def agreement(a, b, sel):
    ea, eb = a["cls"][sel] & 3 == 0, b["cls"][sel] & 3 == 0
    dn = np.abs(a["n"][sel].astype(np.int64) - b["n"][sel].astype(np.int64))
    same = (ea == eb) & (~ea | (dn == 0)) & ((a["cls"][sel] & 3) == (b["cls"][sel] & 3))
    off1 = (ea == eb) & (~ea | (dn <= 1))
    both = ea & eb & (dn == 0)
    rel = np.abs(a["nu"][sel][both] - b["nu"][sel][both]) / np.abs(a["nu"][sel][both])
    return {"count_match": float(same.mean()), "within_one": float(off1.mean()),
            "escape_agreement": float((ea == eb).mean()),
            "nu_rel_err_median": float(np.median(rel)) if rel.size else None,
            "nu_rel_err_p99": float(np.quantile(rel, 0.99)) if rel.size else None}


def run(v, samples, bits_list, seed=11, round_orbit=False):
    job = fdref.make_job(v["re"], v["im"], v["width"], v["nx"], v["ny"], v["max_iter"],
                         escape_radius=v["escape_radius"], columns=fdref.COL_NU, tier=v["tier"])
    ref = fdref.Ref.for_job(job)
    bla = None
    if v["bla"] is not None:
        dc, e = fdref.bla_dc_bound(job)
        bla = fdref.Bla(ref, v["bla"], dc, e)
    n = v["nx"] * v["ny"]
    mask = np.zeros(n, np.uint8)
    pick = np.random.default_rng(seed).choice(n, min(samples, n), replace=False)
    mask[pick] = 1
    sel = mask.astype(bool)
    fdref.set_delta_bits(0)
    t = time.perf_counter()
    base = fdref.render_columns(job, ref, bla, mask=mask)
    out = []
    for bits in bits_list:
        fdref.set_delta_bits(bits, round_orbit=round_orbit)
        try:
            got = fdref.render_columns(job, ref, bla, mask=mask)
        finally:
            fdref.set_delta_bits(0)
        out.append(dict(view=v["name"], samples=int(sel.sum()), delta_bits=bits, orbit_rounded=round_orbit,
                        **agreement(base, got, sel)))
    return out, time.perf_counter() - t


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--samples", type=int, default=20_000)
    ap.add_argument("--bits", type=int, nargs="+", default=[24, 32, 40, 48])
    ap.add_argument("--views", nargs="*", default=None, help="view names (default: all)")
    ap.add_argument("--round-orbit", action="store_true",
                    help="also round the orbit point each plain step multiplies the delta by (an FP32 copy of Z)")
    a = ap.parse_args()
    for v in views():
        if a.views and v["name"] not in a.views:
            continue
        rows, dt = run(v, a.samples, a.bits, round_orbit=a.round_orbit)
        for r in rows:
            print(json.dumps(dict(r, seconds=round(dt, 1))), flush=True)


if __name__ == "__main__":
    main()
