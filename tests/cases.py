"""Small lens configurations shared by the tests (sizes chosen so that the FP64
oracle finishes in seconds)."""
import numpy as np

# IRS, equal masses (the shape of the reference's plain IRS case at reduced size)
IRS_SMALL = dict(kappa_tot=0.4, shear=0.3, kappa_star=0.4, theta_star=1.0, mass_function="equal",
                 half_length_y1=3.0, half_length_y2=3.0, num_pixels_y1=96, num_pixels_y2=96, num_rays_y=16,
                 light_loss=0.01, random_seed=11, write_histograms=0)
# IPM, Salpeter masses with a smooth fraction (shape of the plain IPM case at reduced size)
IPM_SMALL = dict(kappa_tot=0.45, shear=0.4, smooth_fraction=0.5, theta_star=2.31, mass_function="salpeter",
                 m_lower=0.08, m_upper=1.0, half_length_y1=4.0, half_length_y2=4.0, num_pixels_y1=128,
                 num_pixels_y2=128, num_rays_y=1, light_loss=0.01, random_seed=22, write_histograms=0)
# rectangular field with the Taylor-series smooth sheet, Kroupa masses
IPM_RECT = dict(kappa_tot=0.7, shear=0.2, smooth_fraction=0.1, theta_star=1.0, mass_function="kroupa",
                m_lower=0.01, m_upper=1.5, rectangular=True, approx=True, half_length_y1=2.0,
                half_length_y2=2.0, num_pixels_y1=64, num_pixels_y2=64, num_rays_y=1, light_loss=0.01,
                random_seed=33, write_histograms=0)


def lattice(m, vertices: bool):
    """Lattice coordinates as the kernels form them: base + 2 * (rhs * i)."""
    rx, ry = m.value("ray_half_sep_1"), m.value("ray_half_sep_2")
    ox = m.value("center_x1") - m.value("half_length_x1")
    oy = m.value("center_x2") - m.value("half_length_x2")
    nx, ny = int(m.value("num_ray_threads_1")), int(m.value("num_ray_threads_2"))
    if vertices:
        bx, by, nx, ny = ox, oy, nx + 1, ny + 1
    else:
        bx, by = ox + rx, oy + ry
    x = bx + 2.0 * (rx * np.arange(nx, dtype=np.float64))
    y = by + 2.0 * (ry * np.arange(ny, dtype=np.float64))
    return x, y


def oracle_lens(m):
    from oracle import pyoracle as po
    return po.lens(m.kappa_tot, m.shear, m.kappa_star, m.theta_star, int(m.rectangular), int(m.approx),
                   int(m.value("taylor_smooth")), (m.value("corner_x1"), m.value("corner_x2")))


def to_pixels(m, wx, wy):
    """Source position -> pixel units with the row axis flipped (ipm_functions.cuh:159-165)."""
    hx, hy = m.half_length_y1, m.half_length_y2
    npx, npy = m.num_pixels_y1, m.num_pixels_y2
    px = ((wx - m.center_y1) + hx) * npx / (2 * hx)
    py = ((wy - m.center_y2) + hy) * npy / (2 * hy)
    return px, npy - py
