"""Loader and comparator for the frozen mpmath truth pack (tests/golden/truth_v1).

Restates crates/fd-kernel/examples/support/mod.rs of junovhs/fractodactyl: `load`
(:29-117), `load_edges` (:131-168), and `compare` (:235-330) with its 1e-3 output-pixel
displacement gate, 1e-2 relative DE and 1e-3 radian normal raw tolerances.
"""
import gzip
import math
import os

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "truth_v1")
CASES = ["exterior", "extreme", "filament", "parabolic", "period764"]


def load(name):
    with gzip.open(os.path.join(GOLDEN, name + ".tsv.gz"), "rt") as f:
        lines = f.read().splitlines()
    assert lines[0] == "fd-truth\t1"
    v = lines[1].split("\t")
    assert len(v) == 12 and v[0] == "view"
    case = dict(name=v[1], re=v[2], im=v[3], width=v[4], nx=int(v[5]), ny=int(v[6]), ss=int(v[7]),
                max_iter=int(v[8]), escape_radius=float(v[9]), rotation=float(v[10]), bits=int(v[11]))
    points = []
    for line in lines[2:]:
        if line.startswith("#"):
            continue
        f = line.split("\t")
        assert len(f) == 8 and int(f[0]) == len(points)
        points.append((f[1], int(f[2]), [float(x) for x in f[3:]]))
    assert len(points) == case["nx"] * case["ny"]
    case["points"] = points
    return case


def load_edges():
    edges = []
    with open(os.path.join(GOLDEN, "precision-edges.txt")) as f:
        lines = f.read().splitlines()
    assert lines[0] == "fd-truth-edges\t1"
    for line in lines[1:]:
        if line.startswith("#"):
            continue
        f = line.split("\t")
        edges.append(dict(case=f[0], index=int(f[1]), iteration=int(f[8])))
    return edges


def _displacement(excess, rate):
    if excess <= 0.0:
        return 0.0
    return excess / rate if rate > 0.0 else math.inf


def compare(case, cls, nu, de, normal, edges, auto_tier=True):
    """Score one route's columns against the pack (support/mod.rs:235-330)."""
    s = dict(class_mismatches=0, known_edges=0, scalar_failures=0, nu_px=0.0, de_px=0.0, normal_px=0.0,
             mismatched=[])
    edge_idx = {e["index"] for e in edges if e["case"] == case["name"]}
    for i, (truth, it, values) in enumerate(case["points"]):
        kind = int(cls[i]) & 3
        ok = {"E": kind == 0, "A": kind == 1, "U": kind in (1, 2)}[truth]
        if not ok:
            s["class_mismatches"] += 1
            s["mismatched"].append(i)
            if auto_tier and kind == 2 and truth == "E" and i in edge_idx:
                s["known_edges"] += 1
            continue
        if truth != "E":
            continue
        t_nu, t_de, t_angle, de_rate, normal_rate = values
        g_nu, g_de = float(nu[i]), float(de[i])
        g_angle = float(normal[i]) * 2 * math.pi / 65536.0
        if not (math.isfinite(g_nu) and math.isfinite(g_de)):
            s["scalar_failures"] += 1
            continue
        nu_px = abs(g_nu - t_nu) * t_de * math.log(2) / 2.0
        de_diff = abs(g_de - t_de)
        de_px = _displacement(de_diff - t_de * 2.0 ** -24, de_rate) if de_diff / t_de > 1e-2 else 0.0
        nd = abs(math.fmod(g_angle - t_angle + math.pi, 2 * math.pi))
        nd = abs((g_angle - t_angle + math.pi) % (2 * math.pi) - math.pi)
        normal_px = _displacement(nd - math.pi / 65536.0, normal_rate) if nd > 1e-3 else 0.0
        s["nu_px"] = max(s["nu_px"], nu_px)
        s["de_px"] = max(s["de_px"], de_px)
        s["normal_px"] = max(s["normal_px"], normal_px)
        if nu_px > 1e-3 or de_px > 1e-3 or normal_px > 1e-3:
            s["scalar_failures"] += 1
    return s
