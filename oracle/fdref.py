"""ctypes binding of the CPU oracle (liboracle.so, see fdref.h).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg, never by the product package.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")

COL_CLASS, COL_NU, COL_DE, COL_NORMAL, COL_BOUND, COL_STRIPE = 1, 2, 4, 8, 16, 32
TIER = {None: -1, "auto": -1, "f64": 0, "fx": 1, "fixed": 1, "scaled": 2}


class Job(C.Structure):
    _fields_ = [
        ("center_re", C.c_char_p),
        ("center_im", C.c_char_p),
        ("width", C.c_char_p),
        ("rotation", C.c_double),
        ("nx", C.c_uint32),
        ("ny", C.c_uint32),
        ("ss", C.c_uint32),
        ("max_iter", C.c_uint64),
        ("escape_radius", C.c_double),
        ("columns", C.c_uint32),
        ("threads", C.c_int32),
        ("tier", C.c_int32),
        ("row_first", C.c_uint32),
        ("row_step", C.c_uint32),
        ("stripe_window", C.c_uint32),
        ("stripe_freq", C.c_double),
    ]


class Outcome(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("n", C.c_uint64),
        ("zr", C.c_double),
        ("zi", C.c_double),
        ("dr", C.c_double),
        ("di", C.c_double),
        ("dexp", C.c_int64),
        ("blocks", C.c_uint64),
        ("skipped", C.c_uint64),
        ("shift", C.c_double),
        ("ez", C.c_double),
        ("ed", C.c_double),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("reference_len", C.c_uint64),
        ("iterations", C.c_uint64),
        ("blocks", C.c_uint64),
        ("skipped", C.c_uint64),
        ("fallback_samples", C.c_uint64),
        ("closed_form_samples", C.c_uint64),
        ("shift_px", C.c_double),
    ]


class Columns(C.Structure):  # fdref_columns
    _fields_ = [(k, C.c_void_p) for k in ("cls", "nu", "de", "normal", "bound", "n", "z", "dz", "dexp", "ez", "ed",
                                          "stripe")]


class SeriesInfo(C.Structure):
    _fields_ = [(k, C.c_uint64) for k in ("n", "points", "built_steps", "coefficient_pairs", "order",
                                          "growth_count")] + \
               [(k, C.c_double) for k in ("rho", "state_bound", "derivative_bound", "shift_px")] + \
               [("stop", C.c_char * 16)]


def build():
    """Compile liboracle.so from the C++ restatement (make in oracle/)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        P, D, U64, I64, U32, I32 = C.c_void_p, C.c_double, C.c_uint64, C.c_int64, C.c_uint32, C.c_int32
        L.fdref_last_error.restype = C.c_char_p
        L.fdref_plane.argtypes = [C.POINTER(Job), C.POINTER(D), C.POINTER(I64), C.POINTER(I32),
                                  C.POINTER(U64), C.POINTER(D), C.POINTER(D)]
        L.fdref_reference.restype = P
        L.fdref_reference.argtypes = [C.POINTER(Job)]
        L.fdref_reference_f64.restype = P
        L.fdref_reference_f64.argtypes = [D, D, U64, D]
        L.fdref_reference_fixed.restype = P
        L.fdref_reference_fixed.argtypes = [C.c_char_p, C.c_char_p, U64, U64]
        L.fdref_reference_arrays.restype = P
        L.fdref_reference_arrays.argtypes = [P, P, U64, U32]
        L.fdref_ref_len.restype = U64
        L.fdref_ref_len.argtypes = [P]
        L.fdref_ref_bits.restype = U32
        L.fdref_ref_bits.argtypes = [P]
        L.fdref_ref_copy.argtypes = [P, P, P]
        L.fdref_ref_nucleus_period.restype = I64
        L.fdref_ref_nucleus_period.argtypes = [P]
        L.fdref_ref_free.argtypes = [P]
        L.fdref_bla_build.restype = P
        L.fdref_bla_build.argtypes = [P, D, D, I64]
        L.fdref_bla_levels.restype = U32
        L.fdref_bla_levels.argtypes = [P]
        L.fdref_bla_block_count.restype = U64
        L.fdref_bla_block_count.argtypes = [P]
        L.fdref_bla_export.argtypes = [P, P, P]
        L.fdref_bla_find.restype = U64
        L.fdref_bla_find.argtypes = [P, U64, D, U64, C.POINTER(U64), C.POINTER(U64)]
        L.fdref_bla_free.argtypes = [P]
        L.fdref_bla_dc_bound.argtypes = [C.POINTER(Job), C.POINTER(D), C.POINTER(I64)]
        L.fdref_iterate.argtypes = [P, P, C.c_int, C.c_int, C.c_int, D, D, D, D, I64, U64, D, I64,
                                    C.POINTER(Outcome)]
        L.fdref_render.argtypes = [C.POINTER(Job), P, P, P, P, P, P, P, P, P, P, C.POINTER(Stats),
                                   C.c_char_p, C.c_size_t]
        L.fdref_store_escaped.argtypes = [D, I64, U32, D, U64, D, D, D, D, I64,
                                          C.POINTER(D), C.POINTER(C.c_float), C.POINTER(C.c_uint16)]
        L.fdref_direct.restype = U64
        L.fdref_direct.argtypes = [C.c_char_p, C.c_char_p, D, D, I64, U64, U64, D, C.POINTER(D), C.POINTER(D)]
        L.fdref_render_fds.restype = I64
        L.fdref_render_fds.argtypes = [C.POINTER(Job), P, P, P, U64]
        L.fdref_iterate_from.argtypes = [P, P, C.c_int, C.c_int, C.c_int, D, D, D, D, I64, U64, D, I64,
                                         U64, D, D, D, D, C.POINTER(Outcome)]
        L.fdref_iterate_stripe.argtypes = [P, P, C.c_int, C.c_int, D, D, I64, U64, D, I64, C.c_uint32, D,
                                           C.POINTER(Outcome), C.POINTER(C.c_float)]
        L.fdref_series_build.restype = P
        L.fdref_series_build.argtypes = [P, D, D, U64, U64]
        L.fdref_series_get.argtypes = [P, C.POINTER(SeriesInfo), P]
        L.fdref_series_with_n.restype = P
        L.fdref_series_with_n.argtypes = [P, U64]
        L.fdref_series_eval.argtypes = [P, C.c_int, D, D, P]
        L.fdref_series_free.argtypes = [P]
        L.fdref_render_series.argtypes = [C.POINTER(Job), P, P, P, P, P, P, P, P, P, P, P, P, C.POINTER(Stats),
                                          C.c_char_p, C.c_size_t]
        L.fdref_error_radius.argtypes = [P, I64, D, D, P]
        L.fdref_iterate_bounded.argtypes = [P, C.c_int, C.c_int, D, D, D, D, U64, D, I64, D, D, C.POINTER(Outcome)]
        L.fdref_render_columns.argtypes = [C.POINTER(Job), P, P, P, P, C.POINTER(Columns), C.POINTER(Stats),
                                           C.c_char_p, C.c_size_t]
        L.fdref_set_delta_bits.argtypes = [C.c_int, C.c_uint64, C.c_uint64, C.c_int]
        _lib = L
    return _lib


def set_delta_bits(bits, from_n=0, to_n=2 ** 64 - 1, round_orbit=False):
    """Precision experiment (not the reference's algorithm): round every delta the kernel
    writes to `bits` mantissa bits (24: an ideal FP32-mantissa delta) while the iteration
    count it leaves lies in [from_n, to_n); round_orbit: the orbit point each plain step
    multiplies the delta by too (an FP32 copy of Z); 0 restores the reference's binary64
    kernel. Process-wide."""
    if lib().fdref_set_delta_bits(int(bits), int(from_n), int(to_n), int(bool(round_orbit))) != 0:
        raise ValueError(f"delta bits must lie in [0, 52] and from_n <= to_n, got {bits}, {from_n}, {to_n}")


def _err():
    return lib().fdref_last_error().decode()


def make_job(re, im, width, nx, ny, max_iter, rotation=0.0, ss=1, escape_radius=1e10,
             columns=COL_NU | COL_DE | COL_NORMAL, threads=None, tier=None, row_first=0, row_step=1,
             stripe_window=16, stripe_freq=5.0):
    j = Job()
    j._keep = [s.encode() if isinstance(s, str) else s for s in (re, im, width)]
    j.center_re, j.center_im, j.width = j._keep
    j.rotation = rotation
    j.nx, j.ny, j.ss = nx, ny, ss
    j.max_iter = max_iter
    j.escape_radius = escape_radius
    j.columns = columns
    j.threads = threads or os.cpu_count() or 1
    j.tier = TIER[tier] if not isinstance(tier, int) else tier
    j.row_first, j.row_step = row_first, row_step
    j.stripe_window, j.stripe_freq = stripe_window, stripe_freq
    return j


class Ref:
    """A Reference orbit (crates/fd-kernel/src/reference.rs:7-10) held by the oracle."""

    def __init__(self, handle):
        if not handle:
            raise ValueError(_err())
        self.h = handle

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.fdref_ref_free(self.h)
            self.h = None

    @classmethod
    def for_job(cls, job):
        return cls(lib().fdref_reference(C.byref(job)))

    @classmethod
    def f64(cls, cr, ci, max_iter, escape_radius):
        return cls(lib().fdref_reference_f64(cr, ci, max_iter, escape_radius))

    @classmethod
    def fixed(cls, re, im, bits, max_iter):
        return cls(lib().fdref_reference_fixed(re.encode(), im.encode(), bits, max_iter))

    @classmethod
    def arrays(cls, re, im, bits):
        re = np.ascontiguousarray(re, np.float64)
        im = np.ascontiguousarray(im, np.float64)
        return cls(lib().fdref_reference_arrays(re.ctypes.data, im.ctypes.data, len(re), bits))

    def __len__(self):
        return lib().fdref_ref_len(self.h)

    @property
    def bits(self):
        return lib().fdref_ref_bits(self.h)

    def arrays_(self):
        n = len(self)
        re, im = np.empty(n), np.empty(n)
        lib().fdref_ref_copy(self.h, re.ctypes.data, im.ctypes.data)
        return re, im

    def nucleus_period(self):
        p = lib().fdref_ref_nucleus_period(self.h)
        return None if p < 0 else int(p)


class Bla:
    """A BLA table (crates/fd-kernel/src/bla.rs:137-151) built by the oracle."""

    def __init__(self, ref, eps, dc_max, dc_exp=0):
        self.ref = ref
        self.h = lib().fdref_bla_build(ref.h, eps, dc_max, dc_exp)
        if not self.h:
            raise ValueError(_err())

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.fdref_bla_free(self.h)
            self.h = None

    @property
    def levels(self):
        return lib().fdref_bla_levels(self.h)

    def export(self):
        """Level-major blocks as an (N, 7) array and level offsets (levels + 1)."""
        n = lib().fdref_bla_block_count(self.h)
        blocks = np.zeros((n, 7))
        offs = np.zeros(self.levels + 1, np.uint64)
        lib().fdref_bla_export(self.h, blocks.ctypes.data, offs.ctypes.data)
        return blocks, offs

    def find(self, m, d2, budget):
        lv, ix = C.c_uint64(), C.c_uint64()
        n = lib().fdref_bla_find(self.h, m, d2, budget, C.byref(lv), C.byref(ix))
        return None if n == 0 else (int(lv.value), int(ix.value), int(n))


class Series:
    """A parameter-series start (crates/fd-kernel/src/series.rs:57-84) built by the oracle:
    Series::build with SeriesConfig::default() over the oracle orbit `ref`."""

    def __init__(self, ref, rho, pixel, max_iter, stalled_steps=32, _h=None):
        self.ref = ref
        self.h = _h if _h is not None else lib().fdref_series_build(ref.h, rho, pixel, max_iter, stalled_steps)
        if not self.h:
            raise ValueError(_err())

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.fdref_series_free(self.h)
            self.h = None

    def info(self):
        i = SeriesInfo()
        lib().fdref_series_get(self.h, C.byref(i), None)
        d = {k: getattr(i, k) for k, _ in SeriesInfo._fields_}
        d["stop"] = i.stop.decode()
        return d

    def coefficients(self):
        """b[1..order] as an (order, 2) array of (re, im)."""
        i = SeriesInfo()
        lib().fdref_series_get(self.h, C.byref(i), None)
        b = np.zeros((i.order, 2))
        lib().fdref_series_get(self.h, C.byref(i), b.ctypes.data)
        return b

    def with_n(self, n):
        return Series(self.ref, 0, 0, 0, _h=lib().fdref_series_with_n(self.h, n))

    def eval(self, ar, ai, derivative=True):
        out = np.zeros(4)
        lib().fdref_series_eval(self.h, int(derivative), ar, ai, out.ctypes.data)
        return tuple(out)


def render_series(job, ref, series, bla=None, mask=None, raw=False):
    """render_series / Series::render_masked: render() with every sample started from the
    series; mask (nx*ny bytes) renders only the samples where it is nonzero."""
    n = job.nx * job.ny
    cls = np.zeros(n, np.uint8)
    nu = np.zeros(n, np.float64)
    de = np.zeros(n, np.float32)
    normal = np.zeros(n, np.uint16)
    it = np.zeros(n, np.uint64)
    z = np.zeros(2 * n) if raw else None
    dz = np.zeros(2 * n) if raw else None
    dexp = np.zeros(n, np.int64) if raw else None
    m = None if mask is None else np.ascontiguousarray(mask, dtype=np.uint8)
    st = Stats()
    kernel = C.create_string_buffer(256)
    ptr = lambda a: a.ctypes.data if a is not None else None
    rc = lib().fdref_render_series(C.byref(job), ref.h, bla.h if bla else None, series.h, ptr(m), ptr(cls), ptr(nu),
                                   ptr(de), ptr(normal), ptr(it), ptr(z), ptr(dz), ptr(dexp), C.byref(st), kernel,
                                   256)
    if rc != 0:
        raise ValueError(_err())
    out = dict(cls=cls, nu=nu, de=de, normal=normal, n=it, kernel=kernel.value.decode(),
               stats=dict(reference_len=st.reference_len, iterations=st.iterations, blocks=st.blocks,
                          skipped=st.skipped, fallback_samples=st.fallback_samples,
                          closed_form_samples=st.closed_form_samples, shift_px=st.shift_px))
    if raw:
        out.update(z=z.reshape(n, 2), dz=dz.reshape(n, 2), dexp=dexp)
    return out


def error_radius(ref, bits, c_re, c_im):
    """Reference::error_radius (reference.rs:122-148); bits None for an f64 orbit."""
    q = np.zeros(len(ref))
    if lib().fdref_error_radius(ref.h, -1 if bits is None else bits, c_re, c_im, q.ctypes.data) != 0:
        raise ValueError(_err())
    return q


def iterate_bounded(ref, bits, c_re, c_im, c=None, ar=0.0, ai=0.0, max_iter=1000, r2=1e20, derivative=True):
    """The bounded variant of sample.rs:170-581 (B) with the orbit's error radii from
    (bits, c_re, c_im); the result carries the escaped sample's radii ez, ed."""
    o = Outcome()
    rc = lib().fdref_iterate_bounded(ref.h, int(derivative), c is not None, c[0] if c else 0.0, c[1] if c else 0.0,
                                     ar, ai, max_iter, r2, -1 if bits is None else bits, c_re, c_im, C.byref(o))
    if rc != 0:
        raise ValueError(_err())
    kind = {0: "escaped", 1: "interior", 2: "unresolved"}[o.kind]
    return dict(kind=kind, n=o.n, zr=o.zr, zi=o.zi, dr=o.dr, di=o.di, dexp=o.dexp, ez=o.ez, ed=o.ed)


def render_columns(job, ref=None, bla=None, series=None, mask=None):
    """Every output of a render (fdref_render_columns): the columns, the Bound column
    (with COL_BOUND) and the raw state with the error radii of escaped samples."""
    n = job.nx * job.ny
    out = dict(cls=np.zeros(n, np.uint8), nu=np.zeros(n), de=np.zeros(n, np.float32), normal=np.zeros(n, np.uint16),
               bound=np.zeros(n, np.float32), n=np.zeros(n, np.uint64), z=np.zeros((n, 2)), dz=np.zeros((n, 2)),
               dexp=np.zeros(n, np.int64), ez=np.zeros(n), ed=np.zeros(n), stripe=np.zeros(n, np.float32))
    cols = Columns(**{k: v.ctypes.data for k, v in out.items()})
    m = None if mask is None else np.ascontiguousarray(mask, dtype=np.uint8)
    st = Stats()
    kernel = C.create_string_buffer(256)
    rc = lib().fdref_render_columns(C.byref(job), ref.h if ref else None, bla.h if bla else None,
                                    series.h if series else None, m.ctypes.data if m is not None else None,
                                    C.byref(cols), C.byref(st), kernel, 256)
    if rc != 0:
        raise ValueError(_err())
    out["kernel"] = kernel.value.decode()
    out["stats"] = dict(reference_len=st.reference_len, iterations=st.iterations, blocks=st.blocks,
                        skipped=st.skipped, fallback_samples=st.fallback_samples,
                        closed_form_samples=st.closed_form_samples, shift_px=st.shift_px)
    return out


def plane(job):
    hm, he, tier, bits, cr, ci = C.c_double(), C.c_int64(), C.c_int32(), C.c_uint64(), C.c_double(), C.c_double()
    if lib().fdref_plane(C.byref(job), C.byref(hm), C.byref(he), C.byref(tier), C.byref(bits), C.byref(cr),
                         C.byref(ci)) != 0:
        raise ValueError(_err())
    return dict(h_m=hm.value, h_e=he.value, tier=tier.value, bits=bits.value, c_re=cr.value, c_im=ci.value)


def bla_dc_bound(job):
    dc, e = C.c_double(), C.c_int64()
    if lib().fdref_bla_dc_bound(C.byref(job), C.byref(dc), C.byref(e)) != 0:
        raise ValueError(_err())
    return dc.value, e.value


def iterate(ref, bla=None, extended=False, derivative=True, c=None, ar=0.0, ai=0.0, offset_exp=0,
            max_iter=1000, r2=1e20, nucleus=-2, start=None):
    """One sample through sample.rs:170-581. nucleus -2: the orbit's own gate. start:
    (n, xr, xi, dr, di), a state after n iterates to continue from (sample.rs:69-80)."""
    o = Outcome()
    sn, sxr, sxi, sdr, sdi = start if start is not None else (0, 0.0, 0.0, 0.0, 0.0)
    rc = lib().fdref_iterate_from(ref.h, bla.h if bla else None, int(extended), int(derivative), c is not None,
                                  c[0] if c else 0.0, c[1] if c else 0.0, ar, ai, offset_exp, max_iter, r2,
                                  -1 if nucleus is None else nucleus, sn, sxr, sxi, sdr, sdi, C.byref(o))
    if rc != 0:
        raise ValueError(_err())
    kind = {0: "escaped", 1: "interior", 2: "unresolved"}[o.kind]
    return dict(kind=kind, n=o.n, zr=o.zr, zi=o.zi, dr=o.dr, di=o.di, dexp=o.dexp, blocks=o.blocks,
                skipped=o.skipped, shift=o.shift)


def iterate_stripe(ref, bla=None, extended=False, derivative=False, ar=0.0, ai=0.0, offset_exp=0, max_iter=1000,
                   r2=1e20, nucleus=-2, window=16, freq=5.0):
    """One sample from Z_0 with the Stripe recorder (stripe.rs): (outcome dict, stripe value)."""
    o, v = Outcome(), C.c_float()
    rc = lib().fdref_iterate_stripe(ref.h, bla.h if bla else None, int(extended), int(derivative), ar, ai, offset_exp,
                                    max_iter, r2, -1 if nucleus is None else nucleus, window, freq, C.byref(o),
                                    C.byref(v))
    if rc != 0:
        raise ValueError(_err())
    kind = {0: "escaped", 1: "interior", 2: "unresolved"}[o.kind]
    return dict(kind=kind, n=o.n, zr=o.zr, zi=o.zi, blocks=o.blocks, skipped=o.skipped), v.value


def render(job, ref=None, bla=None, raw=False):
    """render_with / render_bla: columns (and raw outcomes) as numpy arrays."""
    n = job.nx * job.ny
    cls = np.zeros(n, np.uint8)
    nu = np.zeros(n, np.float64)
    de = np.zeros(n, np.float32)
    normal = np.zeros(n, np.uint16)
    it = np.zeros(n, np.uint64)
    z = np.zeros(2 * n) if raw else None
    dz = np.zeros(2 * n) if raw else None
    dexp = np.zeros(n, np.int64) if raw else None
    st = Stats()
    kernel = C.create_string_buffer(256)
    ptr = lambda a: a.ctypes.data if a is not None else None
    rc = lib().fdref_render(C.byref(job), ref.h if ref else None, bla.h if bla else None, ptr(cls), ptr(nu),
                            ptr(de), ptr(normal), ptr(it), ptr(z), ptr(dz), ptr(dexp), C.byref(st), kernel, 256)
    if rc != 0:
        raise ValueError(_err())
    out = dict(cls=cls, nu=nu, de=de, normal=normal, n=it, kernel=kernel.value.decode(),
               stats=dict(reference_len=st.reference_len, iterations=st.iterations, blocks=st.blocks,
                          skipped=st.skipped, fallback_samples=st.fallback_samples,
                          closed_form_samples=st.closed_form_samples, shift_px=st.shift_px))
    if raw:
        out.update(z=z.reshape(n, 2), dz=dz.reshape(n, 2), dexp=dexp)
    return out


def store_escaped(h_m, h_e, ss, rotation, n, zr, zi, dr, di, dexp):
    nu, de, nm = C.c_double(), C.c_float(), C.c_uint16()
    lib().fdref_store_escaped(h_m, h_e, ss, rotation, n, zr, zi, dr, di, dexp, C.byref(nu), C.byref(de),
                              C.byref(nm))
    return nu.value, de.value, nm.value


def render_fds(job, ref=None, bla=None):
    size = lib().fdref_render_fds(C.byref(job), ref.h if ref else None, bla.h if bla else None, None, 0)
    if size < 0:
        raise ValueError(_err())
    buf = (C.c_uint8 * size)()
    lib().fdref_render_fds(C.byref(job), ref.h if ref else None, bla.h if bla else None, buf, size)
    return bytes(buf)


def fnv1a64(data):
    h = 0xCBF29CE484222325
    for b in data:
        h = ((h ^ b) * 0x100000001B3) & 0xFFFFFFFFFFFFFFFF
    return h


def direct(cre, cim, ar, ai, oe, bits, max_iter, escape_radius):
    """fd-fixed direct iteration at the sample's exact c: (n or None, zr, zi)."""
    zr, zi = C.c_double(), C.c_double()
    n = lib().fdref_direct(cre.encode(), cim.encode(), ar, ai, oe, bits, max_iter, escape_radius, C.byref(zr),
                           C.byref(zi))
    if n == 2**64 - 1:
        raise ValueError("direct iteration: bad centre")
    return (None if n == 0 else int(n)), zr.value, zi.value
