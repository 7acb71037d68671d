"""Writes KHARMA-format GRMHD dumps (Parthenon .phdf) for tests (test
infrastructure): the layout the reference's KHARMA loader reads
(src/grmhd/kharma_loader.cpp:751-821) and its own synthetic KHARMA fixture
uses -- /Info NumMeshBlocks (int64) and MeshBlockSize (int64[3]: nx1, nx2,
nx3 of a meshblock) and Time, the run's parameter text as the /Input File
string attribute (<parthenon/mesh>, <coordinates>, <GRMHD> blocks),
/Blocks/loc.lx123 (int64 [nblocks][3]), prims.rho and prims.u
[nblocks][nx3][nx2][nx1], prims.uvec and prims.B [nblocks][3][nx3][nx2][nx1]
-- through tests/hdf5_library_layout.py.
"""
from __future__ import annotations

import math

import numpy as np

import hdf5_library_layout as h5w


def parameter_text(model, transform="fmks", extra=""):
    x1max = model.startx1 + model.n1 * model.dx1
    x2max = model.startx2 + model.n2 * model.dx2
    x3max = model.startx3 + model.n3 * model.dx3
    return ("<parthenon/mesh>\n"
            f"nx1 = {model.n1}\nnx2 = {model.n2}\nnx3 = {model.n3}\n"
            f"x1min = {model.startx1:.17g}\nx1max = {x1max:.17g}\n"
            f"x2min = {model.startx2:.17g}\nx2max = {x2max:.17g}\n"
            f"x3min = {model.startx3:.17g}\nx3max = {x3max:.17g}\n"
            "<coordinates>\n"
            f"a = {model.spin:.17g}   # black hole spin\n"
            f"transform = {transform}\n"
            f"r_in = {model.r_in:.17g}\nr_out = {model.r_out:.17g}\n"
            f"hslope = {model.hslope:.17g}\nmks_smooth = {model.mks_smooth:.17g}\n"
            f"poly_alpha = {model.poly_alpha:.17g}\npoly_xt = {model.poly_xt:.17g}\n"
            f"<GRMHD>\ngamma = {model.gam:.17g}\n" + extra)


def write_kharma_dump(path, prims, model, blocks=(2, 2, 1), *, time=100.0, order_seed=0, par=None,
                      profile="earliest", layout="contiguous", chunks=None, filters=(), info_override=None,
                      loc_override=None, dataset_override=None):
    """prims [8, n1, n2, n3] cut into blocks[0] x blocks[1] x blocks[2]
    meshblocks, stored in a seeded shuffled order."""
    n1, n2, n3 = prims.shape[1:]
    b1, b2, b3 = blocks
    m1, m2, m3 = n1 // b1, n2 // b2, n3 // b3
    locs = [(i, j, k) for i in range(b1) for j in range(b2) for k in range(b3)]
    rng = np.random.default_rng(order_seed)
    if order_seed:
        rng.shuffle(locs)
    nmb = len(locs)
    rho = np.empty((nmb, m3, m2, m1), np.float32)
    uu = np.empty_like(rho)
    uvec = np.empty((nmb, 3, m3, m2, m1), np.float32)
    bvec = np.empty_like(uvec)
    for mb, (i, j, k) in enumerate(locs):
        blk = prims[:, i * m1:(i + 1) * m1, j * m2:(j + 1) * m2, k * m3:(k + 1) * m3]  # [8][m1][m2][m3]
        blk = np.transpose(blk, (0, 3, 2, 1))                                        # [8][m3][m2][m1]
        rho[mb], uu[mb] = blk[0], blk[1]
        uvec[mb] = blk[2:5]
        bvec[mb] = blk[5:8]
    root = h5w.Group()
    info = root.group("Info")
    attrs = {"NumMeshBlocks": np.int64(nmb), "MeshBlockSize": np.array([m1, m2, m3], dtype=np.int64),
             "Time": np.float64(time)}
    if info_override:
        attrs.update(info_override)
    for k, v in attrs.items():
        if v is not None:
            info.attr(k, v)
    root.group("Input").attr("File", parameter_text(model) if par is None else par)
    loc = np.array(locs, dtype=np.int64) if loc_override is None else loc_override
    root.group("Blocks").dataset("loc.lx123", loc)
    data = {"prims.rho": rho, "prims.u": uu, "prims.uvec": uvec, "prims.B": bvec}
    if dataset_override:
        data.update(dataset_override)
    for k, v in data.items():
        if v is not None:
            root.dataset(k, v, layout=layout, chunks=(None if chunks is None else chunks[: v.ndim]),
                         filters=filters)
    h5w.write(path, root, profile=profile)
