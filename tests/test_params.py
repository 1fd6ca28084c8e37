"""Host-side parameter derivation (calculate_derived_params, include/ipm.cuh:370-565)
through the C ABI, against the oracle's FP64 restatement, plus input
validation and mass-function moments."""
import math

import numpy as np
import pytest

import irs_b200
from oracle import pyoracle as po

CONFIGS = [
    # C1 plain IRS
    dict(cls="IRS", kappa_tot=0.4, shear=0.3, kappa_star=0.4, theta_star=1.0, mass_function="equal",
         half_length_y1=10, half_length_y2=10, num_pixels_y1=500, num_pixels_y2=500, num_rays_y=100,
         light_loss=0.01),
    # C2 plain IPM at the stated substitute shear 0.4
    dict(cls="IPM", kappa_tot=0.45, shear=0.4, smooth_fraction=0.5, theta_star=2.31, mass_function="salpeter",
         m_lower=0.08, m_upper=1.0, half_length_y1=25, half_length_y2=25, num_pixels_y1=2000, num_pixels_y2=2000,
         num_rays_y=1),
    # C3 rectangular Kroupa field
    dict(cls="IPM", kappa_tot=0.7, shear=0.2, smooth_fraction=0.1, theta_star=1.0, mass_function="kroupa",
         m_lower=0.01, m_upper=1.5, rectangular=True, half_length_y1=50, half_length_y2=50, num_pixels_y1=8192,
         num_pixels_y2=8192, num_rays_y=1),
    # C5 learned-adaptive IPM field
    dict(cls="IPM", kappa_tot=0.6, shear=0.3, smooth_fraction=0.3, theta_star=1.0, mass_function="salpeter",
         m_lower=0.08, m_upper=1.0, half_length_y1=30, half_length_y2=30, num_pixels_y1=4096, num_pixels_y2=4096,
         num_rays_y=1),
    # off-centre, rectangular pixels
    dict(cls="IPM", kappa_tot=0.3, shear=0.25, kappa_star=0.2, theta_star=1.3, mass_function="uniform",
         m_lower=0.1, m_upper=2.0, center_y1=1.5, center_y2=-2.0, half_length_y1=5, half_length_y2=3,
         num_pixels_y1=300, num_pixels_y2=200, num_rays_y=4),
]


def make(cfg, dbl):
    c = dict(cfg)
    cls = getattr(irs_b200, c.pop("cls"))
    return cls(is_double=dbl, **c)


@pytest.mark.parametrize("cfg", CONFIGS)
def test_derived_matches_oracle_fp64(cfg):
    m = make(cfg, True)
    m.derive()
    o = po.derive(m.kappa_tot, m.shear, m.kappa_star, m.theta_star, m.value("mean_mass"), m.value("mean_mass2"),
                  m.light_loss, int(m.rectangular), m.safety_scale, m.center, m.half_length, m.num_pixels,
                  m.num_rays_y)
    for k in ["num_stars", "num_ray_threads_1", "num_ray_threads_2"]:
        assert m.value(k) == o[k], k
    for k, v in o.items():
        assert math.isclose(m.value(k), v, rel_tol=1e-13, abs_tol=1e-300), k


@pytest.mark.parametrize("cfg", CONFIGS)
def test_float_derivation_close_to_double(cfg):
    a, b = make(cfg, False), make(cfg, True)
    a.derive()
    b.derive()
    assert abs(a.value("num_stars") - b.value("num_stars")) <= max(1, 1e-5 * b.value("num_stars"))
    for k in ["num_ray_threads_1", "num_ray_threads_2"]:
        assert abs(a.value(k) - b.value(k)) <= 2
    assert math.isclose(a.value("half_length_x1"), b.value("half_length_x1"), rel_tol=1e-5)


def test_config2_as_published_is_degenerate():
    # kappa = 0.45, shear = 0.55 makes 1 - kappa - shear = 0: the shooting
    # region is unbounded (the reference divides by zero at ipm.cuh:461).
    m = irs_b200.IPM(kappa_tot=0.45, shear=0.55, smooth_fraction=0.5, mass_function="salpeter", m_lower=0.08,
                     m_upper=1.0, theta_star=2.31, half_length_y1=25, half_length_y2=25, num_pixels_y1=2000,
                     num_pixels_y2=2000, is_double=True)
    with pytest.raises(ValueError):
        m.derive()


@pytest.mark.parametrize("bad", [dict(light_loss=0.02), dict(safety_scale=1.05), dict(num_rays_y=0),
                                 dict(num_pixels_y1=0), dict(half_length_y1=-1.0), dict(kappa_star=0.6),
                                 dict(mass_function="nope")])
def test_python_setters_validate(bad):
    args = dict(kappa_tot=0.5, shear=0.2, kappa_star=0.3)
    args.update(bad)
    with pytest.raises(ValueError):
        irs_b200.IPM(**args)


def test_c_validation_rejects_bad_flags():
    m = irs_b200.IPM(kappa_tot=0.5, shear=0.2, kappa_star=0.3)
    m.lib.set_write_maps(m.obj, 3)
    with pytest.raises(ValueError):
        m.derive()
    m.lib.set_write_maps(m.obj, 1)
    m.lib.set_approx(m.obj, 2)
    with pytest.raises(ValueError):
        m.derive()


def _pdf_moments(pdf, lo, hi):
    x = np.logspace(np.log10(lo), np.log10(hi), 400001)
    p = pdf(x)
    z = np.trapezoid(p, x)
    return (np.trapezoid(p * x, x) / z, np.trapezoid(p * x * x, x) / z,
            np.trapezoid(p * x * x * np.log(x), x) / z)


@pytest.mark.parametrize("mf,lo,hi", [("salpeter", 0.08, 1.0), ("kroupa", 0.01, 1.5), ("kroupa", 0.1, 0.4),
                                      ("kroupa", 0.6, 2.0), ("uniform", 0.1, 2.0), ("optical_depth", 0.2, 1.0)])
def test_mass_function_moments(mf, lo, hi):
    m = irs_b200.IPM(kappa_tot=0.5, shear=0.1, kappa_star=0.3, mass_function=mf, m_lower=lo, m_upper=hi,
                     is_double=True, half_length_y1=2, half_length_y2=2, num_pixels_y1=10, num_pixels_y2=10)
    m.derive()
    if mf == "optical_depth":
        ref = (2 * lo * hi / (lo + hi), lo * hi, lo * hi * (lo * np.log(lo) + hi * np.log(hi)) / (lo + hi))
    else:
        def pdf(x):
            if mf == "salpeter":
                return x ** -2.35
            if mf == "uniform":
                return np.ones_like(x)
            m0, m1 = 0.08, 0.5
            return np.where(x < m0, (x / m0) ** -0.3,
                            np.where(x < m1, (x / m0) ** -1.3, (m1 / m0) ** -1.3 * (x / m1) ** -2.3))
        ref = _pdf_moments(pdf, lo, hi)
    got = (m.value("mean_mass"), m.value("mean_mass2"), m.value("mean_mass2_ln_mass"))
    for g, r in zip(got, ref):
        assert math.isclose(g, r, rel_tol=2e-6, abs_tol=1e-9)
