"""Generate golden vectors from the reference's own code compiled for the host.

Run from the repository root after `make -C oracle ref` (needs the reference
sources): python tests/golden/make_golden.py
Writes tests/golden/ref_small.npz with, for a fixed small star field:
  * the reference tree summary (levels, nodes, leaves, star counts);
  * source positions w at sample points (complex_image_to_source);
  * the reference IPM map (shoot_cells_kernel) and IRS map (shoot_rays_kernel)
    for small lattices, and the reference deposition of a fixed corner lattice.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle import pyoracle as po  # noqa: E402


def lattice_params(kappa, gamma, kstar, theta, m2_over_m, light_loss, hly, npix, nry):
    """calculate_derived_params (include/ipm.cuh:437-470) for a given field, double."""
    nrx = 1.0 * nry * npix * npix / (2 * hly * 2 * hly)
    rhs = 1.0 / (2 * np.sqrt(nrx))
    t = theta * np.sqrt(kstar * m2_over_m / light_loss)
    hx, hy = (hly + t) / abs(1 - kappa + gamma), (hly + t) / abs(1 - kappa - gamma)
    n1, n2 = int(hx / (2 * rhs)) + 1, int(hy / (2 * rhs)) + 1
    return rhs, (2 * n1, 2 * n2), (2 * rhs * n1, 2 * rhs * n2)


def main():
    rng = np.random.default_rng(12345)
    n, R = 1200, 36.0
    r = R * np.sqrt(rng.random(n))
    a = 2 * np.pi * rng.random(n)
    m = rng.uniform(0.1, 1.0, n)
    stars = np.stack([r * np.cos(a), r * np.sin(a), m], 1)
    kappa, gamma, kstar, theta = 0.45, 0.4, 0.225, 1.5
    L = po.lens(kappa, gamma, kstar, theta)
    order = 12
    t = po.RefTree(stars, 1.1 * R, order=order, kind="ipm")
    ints, geom, *_ = t.nodes()
    pts = rng.uniform(-8, 8, (4000, 2))
    wx, wy = t.points(L, pts[:, 0], pts[:, 1])
    # IPM map through the reference kernel
    hly, npix = 2.0, 48
    rhs, nrt, hlx = lattice_params(kappa, gamma, kstar, theta, 1.0, 0.01, hly, npix, 1)
    ipm = t.shoot(L, (rhs, rhs), nrt, (0.0, 0.0), hlx, (0.0, 0.0), (hly, hly), (npix, npix))
    # IRS map through the reference kernel
    ti = po.RefTree(stars, 1.1 * R, order=order, kind="irs")
    rhs_i, nrt_i, hlx_i = lattice_params(kappa, gamma, kstar, theta, 1.0, 0.01, hly, npix, 9)
    irs = ti.shoot(L, (rhs_i, rhs_i), nrt_i, (0.0, 0.0), hlx_i, (0.0, 0.0), (hly, hly), (npix, npix), ints=True)
    # reference deposition of a fixed corner lattice
    v = np.stack(np.meshgrid(np.linspace(-3, 30, 41), np.linspace(-2, 28, 37)), -1)
    v = v + rng.normal(0, 0.6, v.shape)
    dep = po.ref_deposit_cells(v, 0.75, (24, 20))
    np.savez_compressed(
        os.path.join(HERE, "ref_small.npz"), stars=stars, lens=np.array([kappa, gamma, kstar, theta]), order=order,
        root_hl=1.1 * R, levels=t.levels, num_nodes=t.n, node_level=ints[:, 0], node_numstars=ints[:, 1],
        node_children=ints[:, 2], node_geom=geom, pts=pts, wx=wx, wy=wy, ipm_hly=hly, ipm_npix=npix, ipm_rhs=rhs,
        ipm_nrt=np.array(nrt), ipm_hlx=np.array(hlx), ipm_map=ipm, irs_rhs=rhs_i, irs_nrt=np.array(nrt_i),
        irs_hlx=np.array(hlx_i), irs_map=irs, dep_verts=v, dep_factor=0.75, dep_map=dep)
    print("wrote", os.path.join(HERE, "ref_small.npz"), "levels", t.levels, "nodes", t.n)


if __name__ == "__main__":
    main()
