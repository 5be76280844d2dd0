"""A zoom film on the CUDA route written as .fds files (fractodactyl_b200.film): every
frame's file equals, byte for byte, the oracle's .fds render of that frame over the same
shared orbit and per-frame BLA table (header, class, nu, de and normal), across the Fixed
and Scaled tiers of a 1e-10 -> 1e-500 film (the first frame without a table)."""
import dataclasses

import pytest

import fdref
import fractodactyl_b200 as fd
from fractodactyl_b200 import film, locations, workloads

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    d = fd.Device(0)
    yield d
    d.close()


def test_film_fds_bytes_equal_oracle(dev, tmp_path):
    frames = [dataclasses.replace(f, params=dataclasses.replace(f.params, nx=48, ny=27))
              for f in (locations.config4()[k] for k in (0, 20, 40, 59))]
    datas = film.render_film(dev, frames, out_dir=str(tmp_path), suffix="")
    assert sorted(p.name for p in tmp_path.iterdir()) == [f"frame_{k:04d}.fds" for k in range(4)]
    assert (tmp_path / "frame_0003.fds").read_bytes() == datas[3]
    # the orbit and tables render_film used, rebuilt the same way for the oracle
    js = workloads.film(dev, frames)
    js.free(dev)
    r = js.refs[0]
    ref = fdref.Ref.arrays(r.re, r.im, r.bits)
    assert len({t for t in js.tiers}) >= 2
    for f, tier, table, data in zip(frames, js.tiers, js.blas, datas):
        t = fdref.Bla(ref, f.bla_eps, table.dc_max, table.dc_exp) if table is not None else None
        v, p = f.view, f.params
        job = fdref.make_job(v.center_re, v.center_im, v.width, p.nx, p.ny, p.max_iter, rotation=v.rotation,
                             ss=p.ss, escape_radius=p.escape_radius, tier=tier)
        assert data == fdref.render_fds(job, ref, t), v.width
    # the route's own files carry its kernel suffix
    tagged = film.render_film(dev, frames[:1])
    assert tagged[0] != datas[0] and film.ROUTE_SUFFIX.encode() in tagged[0]
