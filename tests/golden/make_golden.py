"""Generate the committed golden fixtures from the reference checkout.

Runs only where the reference tree is present (it is not on GPU machines); the outputs
under tests/golden/ are what the tests read. Sources, all from junovhs/fractodactyl:

  truth_v1/*.tsv.gz, precision-edges.txt   bench/truth/v1 (frozen mpmath observations)
  kats.json                                constants of crates/fd-kernel/src/sample.rs tests
                                           (v0 centre :944-947, FNV cases :717-722) and the
                                           k=7676 rung of tools/research/misiurewicz/ladder_rungs.txt,
                                           and the series frames (centre, width) of
                                           docs/2026-10-20/series-frames/results/frames.txt, which
                                           crates/fd-kernel/src/series.rs tests read, and the
                                           mpmath orbit point of crates/fd-fixed/tests/fixtures/v0_orbit.txt
                                           (c, period, z_period and z/dz at 400 digits)
  kern05.json                              per-frame digests of crates/fd-kernel/fixtures/KERN-05.bundle
                                           (format: crates/fd-kernel/examples/kernel_contract.rs:82-96)
                                           plus the bench/locations.txt rows that produced them

usage: python tests/golden/make_golden.py REFERENCE_ROOT
"""
import gzip
import json
import os
import shutil
import struct
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def fnv1a64(data):
    h = 0xCBF29CE484222325
    for b in data:
        h = ((h ^ b) * 0x100000001B3) & 0xFFFFFFFFFFFFFFFF
    return h


def main(root):
    out = os.path.join(HERE, "truth_v1")
    os.makedirs(out, exist_ok=True)
    src = os.path.join(root, "bench", "truth", "v1")
    for name in sorted(os.listdir(src)):
        path = os.path.join(src, name)
        if name.endswith(".tsv"):
            with open(path, "rb") as f, gzip.GzipFile(os.path.join(out, name + ".gz"), "wb", mtime=0) as g:
                g.write(f.read())
        elif name == "precision-edges.txt":
            shutil.copy(path, os.path.join(out, name))

    sample_rs = open(os.path.join(root, "crates/fd-kernel/src/sample.rs")).read()
    v0 = sample_rs.split("const V0: (&str, &str) = (")[1].split(");")[0]
    v0 = [s.strip().strip('"') for s in v0.split(",") if s.strip()]
    fnv = []
    block = sample_rs.split("let cases = [")[1].split("];")[0]
    for line in block.strip().splitlines():
        parts = [p.strip().strip('()"') for p in line.strip().rstrip(",").split(",")]
        fnv.append({"re": parts[0], "im": parts[1], "width": parts[2], "fnv": parts[3]})
    rung = None
    for line in open(os.path.join(root, "tools/research/misiurewicz/ladder_rungs.txt")):
        if line.startswith("7676 "):
            f = line.split()
            rung = {"k": 7676, "period": int(f[1]), "re": f[2], "im": f[3]}
    series_frames = []
    for line in open(os.path.join(root, "docs/2026-10-20/series-frames/results/frames.txt")):
        if line.startswith("#") or not line.strip():
            continue
        f = line.split()
        series_frames.append({"re": f[0], "im": f[1], "width": f[2]})
    v0_orbit = {}
    for line in open(os.path.join(root, "crates/fd-fixed/tests/fixtures/v0_orbit.txt")):
        if line.startswith("#") or not line.strip():
            continue
        f = line.split()
        v0_orbit[f[0]] = f[1:] if len(f) > 2 else f[1]
    kats = {"v0": {"re": v0[0], "im": v0[1]}, "fnv_views": fnv, "rung_7676": rung, "series_frames": series_frames,
            "v0_orbit": v0_orbit}
    with open(os.path.join(HERE, "kats.json"), "w") as f:
        json.dump(kats, f, indent=1)

    locations = []
    for line in open(os.path.join(root, "bench/locations.txt")):
        if line.strip() and not line.startswith("#"):
            f = line.split()
            nx, ny = f[5].split("x")
            locations.append({"name": f[0], "re": f[1], "im": f[2], "width": f[3], "iter": int(f[4]),
                              "nx": int(nx), "ny": int(ny), "rotation": float(f[6]), "tier": f[7]})
    locations.append({"name": "rung-7676", "re": rung["re"], "im": rung["im"], "width": "5.05e-997",
                      "iter": 150000, "nx": 96, "ny": 54, "rotation": 0.0, "tier": "auto"})
    data = open(os.path.join(root, "crates/fd-kernel/fixtures/KERN-05.bundle"), "rb").read()
    magic = b"KERN05-FDS-1\0"
    assert data.startswith(magic)
    pos, frames = len(magic), []
    while pos < len(data):
        (nlen,) = struct.unpack_from("<Q", data, pos)
        name = data[pos + 8:pos + 8 + nlen].decode()
        pos += 8 + nlen
        (blen,) = struct.unpack_from("<Q", data, pos)
        body = data[pos + 8:pos + 8 + blen]
        pos += 8 + blen
        minor = struct.unpack_from("<H", body, 10)[0]
        norm = bytearray(body)
        norm[10:12] = b"\0\0"
        # column offsets: header is padded to 8; class is 1 byte per sample.
        cols, nx, ny = struct.unpack_from("<III", body, 12)
        p = 56
        strs = []
        for _ in range(4):
            (n,) = struct.unpack_from("<H", body, p)
            strs.append(body[p + 2:p + 2 + n].decode())
            p += 2 + n
        hdr = (p + 7) & ~7
        cls = body[hdr:hdr + nx * ny]
        frames.append({"name": name, "bytes": blen, "minor": minor, "fnv_minor0": "0x%016x" % fnv1a64(norm),
                       "kernel": strs[3], "header_bytes": hdr, "class_fnv": "0x%016x" % fnv1a64(cls),
                       "classes": [cls.count(0), cls.count(1), cls.count(2)]})
    with open(os.path.join(HERE, "kern05.json"), "w") as f:
        json.dump({"locations": locations, "frames": frames}, f, indent=1)
    print("wrote truth_v1/, kats.json, kern05.json")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {sys.argv[0]} REFERENCE_CHECKOUT (the junovhs/fractodactyl source tree)")
    main(sys.argv[1])
