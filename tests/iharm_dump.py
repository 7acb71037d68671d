"""Writes iharm-format GRMHD dumps for tests (test infrastructure): the
datasets an iharm dump carries and the reference's iharm loader reads
(src/grmhd/iharm_loader.cpp:254-370): /header/{n1,n2,n3} (int32), /header/a,
/header/gam (or gamma), /header/geom/{startx1..3, dx1..3} and
/header/geom/{fmks|mmks}/{hslope, mks_smooth, poly_alpha, poly_xt, r_in,
r_out} (float64 scalars), /prims [n1][n2][n3][nprim] and the dump time /t,
through tests/hdf5_library_layout.py (the HDF5 library's own structures).
"""
from __future__ import annotations

import numpy as np

import hdf5_library_layout as h5w


def write_iharm_dump(path, prims, model, *, time=100.0, profile="earliest", geom="fmks", gamma_key="gam",
                     layout="contiguous", chunks=None, filters=(), dtype=np.float32, extra_prims=0,
                     time_key="t", prims_override=None, header_override=None):
    """prims: [8, n1, n2, n3] (the library's layout); the file holds
    [n1][n2][n3][8 + extra_prims] of `dtype` (extra fields seeded)."""
    p = np.moveaxis(np.asarray(prims), 0, -1)
    if extra_prims:
        rng = np.random.default_rng(3)
        p = np.concatenate([p, rng.uniform(0.0, 1.0, size=p.shape[:3] + (extra_prims,)).astype(p.dtype)], axis=-1)
    p = np.ascontiguousarray(p, dtype=dtype)
    if prims_override is not None:
        p = prims_override
    root = h5w.Group()
    hdr = root.group("header")
    fields = {"n1": np.int32(model.n1), "n2": np.int32(model.n2), "n3": np.int32(model.n3),
              "a": np.float64(model.spin), gamma_key: np.float64(model.gam)}
    if header_override:
        fields.update(header_override)
    for k, v in fields.items():
        hdr.dataset(k, v)
    if time_key == "header/t":
        hdr.dataset("t", np.float64(time))
    g = hdr.group("geom")
    for k in ("startx1", "startx2", "startx3", "dx1", "dx2", "dx3"):
        g.dataset(k, np.float64(getattr(model, k)))
    m = g.group(geom)
    for k in ("hslope", "mks_smooth", "poly_alpha", "poly_xt", "r_in", "r_out"):
        m.dataset(k, np.float64(getattr(model, k)))
    root.dataset("prims", p, layout=layout, chunks=chunks, filters=filters)
    if time_key == "t":
        root.dataset("t", np.float64(time))
    h5w.write(path, root, profile=profile)
