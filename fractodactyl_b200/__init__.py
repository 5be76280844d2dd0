"""fractodactyl_b200: the per-pixel perturbation hot path of fractodactyl on B200 (sm_100a).

The CUDA library (libfdcuda.so, C ABI in include/fdcuda.h and include/fdhost.h) holds
the kernels and the host set-up; this package is the Python mirror of the reference's
route interface over it (route.py) plus the .fds v1 writer (fds.py).
"""
from .route import (EPS, EPS_MAX, FILM_EPS, Bla, BlaStats, Declined, Device, DeviceTable, Header, Incomplete, Params, Plane,
                    Reference, RouteError, RouteReport, Samples, Series, Stats, View, bla_dc_bound, device, enabled, reference,
                    render, render_bla, render_series, render_with)

__all__ = ["EPS", "EPS_MAX", "FILM_EPS", "Bla", "BlaStats", "Declined", "Device", "DeviceTable", "Header", "Incomplete", "Params",
           "Plane", "Reference", "RouteError", "RouteReport", "Samples", "Series", "Stats", "View", "bla_dc_bound", "device",
           "enabled",
           "reference", "render", "render_bla", "render_series", "render_with"]
