"""The B200 engine against the reference's own GPU code on the same inputs.

The reference (weisluke/irs) is built from its sources for sm_100a into
oracle/_ref/gpu by `make -C oracle refgpu` (its own `compile` flags plus the
B200 target) and driven through its unchanged Python package
(`microlensing.IPM.IPM`) or its `irs_gpu` tool, each run in a child process
(oracle/ref_gpu.py). What is compared:

  * same seed: the star field (curand XORWOW, star.cuh:40-107; mass draws
    mass_functions/*.cuh), the star-field moments and every derived parameter
    the reference writes to `ipm_parameter_info.txt` (calculate_derived_params,
    ipm.cuh:370-565; calculate_star_params, star.cuh:124-161). Double builds:
    identical stars and parameters. Float builds: the reference is compiled
    with --use_fast_math, whose cos/sin/pow approximations move a float star
    by up to 1e-5 of the field radius and a mass by up to 1e-5 relative; the
    integer parameters are still identical and the float ones agree to 1e-5.
  * same star field (the reference's own, read back from its star file):
    IPM maps at the plain-IPM configuration (2000^2, 37 521 stars, 87.6 M
    cells) and IRS maps at the plain-IRS configuration (500^2, 61.7 M rays).
    FP64: IPM median relative error <= 1e-8, 99th percentile <= 1e-7; IRS
    maps identical up to 10 rays. FP32 (against the reference's FP64 map):
    IPM median relative error <= 1e-3 and not above the reference's own FP32
    build's; IRS rays moved <= 1e-3 of those received.
  * the reference's unchanged Python wrapper over this build's lib_ipm.so /
    lib_ipm_double.so placed at its bin/ (lib_ipm.py:5): the same maps as this
    package's own wrapper, bit for bit.
"""
import os
import shutil
import subprocess
import sys

import numpy as np
import pytest

import irs_b200
from oracle import ref_gpu as rg
from tests.cases import IPM_SMALL

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
needs_ref = pytest.mark.skipif(not rg.available("ipm"), reason="the reference's GPU build (oracle/_ref/gpu) is absent")
needs_ref_irs = pytest.mark.skipif(not rg.available("irs"), reason="the reference's irs_gpu build is absent")

INT_KEYS = ("num_stars", "num_pixels_y1", "num_pixels_y2", "num_ray_threads_1", "num_ray_threads_2",
            "expansion_order", "tree_levels", "random_seed", "num_rays_y")
SKIP_KEYS = ("t_shoot_cells", "t_shoot_rays")


def headline_params():
    """The plain-IPM configuration: Salpeter 0.08-1 with theta_star the Einstein
    radius of the mean mass, kappa 0.45, shear 0.40 (the stated substitute for
    0.55), smooth fraction 0.5, 2000^2 pixels over half length 25, seed 2."""
    p = irs_b200.IPM(kappa_tot=0.45, shear=0.4, smooth_fraction=0.5, mass_function="salpeter", m_lower=0.08,
                     m_upper=1.0, theta_star=1.0, is_double=True)
    p.derive()
    theta = float(1.0 / np.sqrt(p.value("mean_mass")))
    p.close()
    return dict(kappa_tot=0.45, shear=0.40, smooth_fraction=0.5, mass_function="salpeter", m_lower=0.08,
                m_upper=1.0, theta_star=theta, half_length_y1=25.0, half_length_y2=25.0, num_pixels_y1=2000,
                num_pixels_y2=2000, num_rays_y=1, random_seed=2, write_histograms=0)


IRS_CASE1 = dict(kappa_tot=0.4, shear=0.3, kappa_star=0.4, theta_star=1.0, mass_function="equal",
                 half_length_y1=10.0, half_length_y2=10.0, num_pixels_y1=500, num_pixels_y2=500, num_rays_y=100,
                 light_loss=0.01, random_seed=1, write_histograms=0)


def rel_err(got, ref):
    ok = ref > 0
    r = np.abs(got[ok].astype(np.float64) - ref[ok].astype(np.float64)) / ref[ok]
    return float(np.median(r)), float(np.quantile(r, 0.99)), float(r.max())


def _sorted(s):
    s = np.asarray(s, np.float64)
    return s[np.lexsort((s[:, 2], s[:, 1], s[:, 0]))]


def _match(a, b):
    """Distance from every star of a to the nearest star of b (positions), and
    the relative mass difference of that pair."""
    from scipy.spatial import cKDTree
    d, i = cKDTree(b[:, :2]).query(a[:, :2])
    return d, np.abs(a[:, 2] - b[i, 2]) / a[:, 2]


SEED_CASES = [
    dict(mass_function="equal", rectangular=False),
    dict(mass_function="uniform", m_lower=0.1, m_upper=2.0, rectangular=True),
    dict(mass_function="salpeter", m_lower=0.08, m_upper=1.0, rectangular=False),
    dict(mass_function="kroupa", m_lower=0.01, m_upper=1.5, rectangular=True, approx=True),
    dict(mass_function="kroupa", m_lower=0.01, m_upper=1.5, rectangular=False),
    dict(mass_function="optical_depth", m_lower=0.2, m_upper=1.0, rectangular=False),
]


@needs_ref
@pytest.mark.parametrize("dbl", [True, False], ids=["double", "float"])
@pytest.mark.parametrize("case", SEED_CASES, ids=lambda c: f"{c['mass_function']}-{'rect' if c['rectangular'] else 'circ'}")
def test_same_seed_stars_and_parameters(gpu, tmp_path, case, dbl):
    p = dict(kappa_tot=0.6, shear=0.25, smooth_fraction=0.3, theta_star=1.0, half_length_y1=3.0,
             half_length_y2=3.0, num_pixels_y1=64, num_pixels_y2=64, num_rays_y=2, random_seed=77,
             write_stars=1, write_maps=0, write_histograms=0, **case)
    rd = tmp_path / "ref"
    rd.mkdir()
    r = rg.run_ipm(p, is_double=dbl, outdir=str(rd))
    m = irs_b200.IPM(**p, is_double=dbl, outfile_prefix=str(tmp_path / "ours_"))
    m.run()
    m.save()
    ours = rg.read_param_info(str(tmp_path / "ours_ipm_parameter_info.txt"))
    ri = r["param_info"]
    for k, v in ri.items():
        if k in SKIP_KEYS or isinstance(v, str):
            continue
        assert k in ours, k
        if k in INT_KEYS or dbl:
            assert ours[k] == v, (k, ours[k], v)
        else:
            assert abs(ours[k] - v) <= 1e-5 * max(abs(v), 1e-3), (k, ours[k], v)
    a, b = _sorted(r["stars"]), _sorted(m.stars)
    assert a.shape == b.shape
    if dbl:
        np.testing.assert_array_equal(a, b)
    else:
        scale = max(abs(ri.get("corner_x1", 0.0)), abs(ri.get("corner_x2", 0.0)), ri.get("rad", 0.0))
        d, dm = _match(a, b)
        assert d.max() <= 1e-5 * scale
        assert dm.max() <= 1e-5
    # the star file the reference wrote reads back as this build's star field
    st, rect, corner, theta = rg.read_starfile(str(rd / "ipm_stars.bin"))
    assert rect == int(case["rectangular"]) and st.shape == a.shape
    m.close()


@pytest.fixture(scope="module")
def headline_ref(tmp_path_factory):
    """The reference's IPM at the plain-IPM configuration (seed 2), float and
    double builds, with its star field written to a star file."""
    if not rg.available("ipm"):
        pytest.skip("the reference's GPU build (oracle/_ref/gpu) is absent")
    td = tmp_path_factory.mktemp("headline")
    p = headline_params()
    out = {}
    gen = rg.run_ipm({**p, "write_stars": 1, "write_maps": 0}, is_double=True, outdir=str(td))
    sf = str(td / "ipm_stars.bin")
    # the reference's own star field, as a star file: both builds of both codes read it
    q = {k: v for k, v in p.items() if k not in ("random_seed", "theta_star", "mass_function", "m_lower", "m_upper",
                                                 "smooth_fraction")}
    q.update(starfile=sf, safety_scale=1.3)  # a drawn field meets the 1.37 coverage check only to sampling noise
    for dbl in (True, False):
        out[dbl] = rg.run_ipm(q, is_double=dbl)
    return q, out, gen


@needs_ref
def test_headline_ipm_fp64_matches_reference(gpu, headline_ref):
    q, ref, _ = headline_ref
    m = irs_b200.IPM(**q, is_double=True)
    m.run()
    med, p99, mx = rel_err(m.magnifications, ref[True]["magnifications"])
    print(f"FP64 vs reference FP64: median {med:.3e} p99 {p99:.3e} max {mx:.3e}")
    assert med <= 1e-8 and p99 <= 1e-7
    m.close()


@needs_ref
def test_headline_ipm_fp32_accuracy_vs_reference(gpu, headline_ref):
    q, ref, _ = headline_ref
    m = irs_b200.IPM(**q, is_double=False)
    m.run()
    truth = ref[True]["magnifications"]
    med, p99, mx = rel_err(m.magnifications, truth)
    rmed, rp99, rmx = rel_err(ref[False]["magnifications"], truth)
    print(f"FP32 vs reference FP64: median {med:.3e} p99 {p99:.3e} max {mx:.3e}; "
          f"reference FP32 vs its FP64: median {rmed:.3e} p99 {rp99:.3e} max {rmx:.3e}")
    assert med <= 1e-3
    assert med <= rmed
    m.close()


@needs_ref_irs
@pytest.mark.parametrize("dbl", [True, False], ids=["double", "float"])
def test_irs_case1_matches_reference_same_stars(gpu, tmp_path, dbl):
    gd = tmp_path / "gen"
    gd.mkdir()
    gen = rg.run_irs({**IRS_CASE1, "write_stars": 1}, str(gd), is_double=True)
    q = {k: v for k, v in IRS_CASE1.items() if k not in ("random_seed", "theta_star", "mass_function", "kappa_star")}
    q.update(starfile=str(gd / "irs_stars.bin"), safety_scale=1.3)
    rd = tmp_path / "ref"
    rd.mkdir()
    r = rg.run_irs(q, str(rd), is_double=dbl)
    m = irs_b200.IRS(**q, is_double=dbl)
    m.run()
    a, b = r["magnifications"].astype(np.int64), m.magnifications.astype(np.int64)
    assert int(r["param_info"]["expansion_order"]) == m.expansion_order
    moved = np.abs(a - b).sum() // 2
    print(f"IRS {'FP64' if dbl else 'FP32'} vs the reference's same build: {moved} of {a.sum()} rays moved")
    if dbl:
        assert moved <= 10
    else:
        assert moved <= 1e-3 * a.sum()
    m.close()


@needs_ref
def test_unchanged_reference_wrapper_over_this_library(gpu, tmp_path):
    """The reference's microlensing package, unchanged, with this build's
    libraries at its bin/ (the drop-in of lib_ipm.py:5)."""
    pkg = tmp_path / "pkg"
    shutil.copytree(os.path.join(rg.REFGPU, "microlensing"), pkg / "microlensing")
    (pkg / "bin").mkdir()
    for lib in ("lib_ipm.so", "lib_ipm_double.so"):
        os.symlink(os.path.join(ROOT, "irs_b200", "lib", lib), pkg / "bin" / lib)
    cfg = {k: v for k, v in IPM_SMALL.items()}
    script = (
        "import sys, numpy as np\n"
        f"sys.path.insert(0, {str(pkg)!r})\n"
        "from microlensing.IPM.ipm import IPM\n"
        "out = {}\n"
        "for dbl in (False, True):\n"
        f"    m = IPM(**{cfg!r}, is_double=dbl, write_maps=0, write_stars=0)\n"
        "    m.run()\n"
        "    out[f'mu{int(dbl)}'] = m.magnifications\n"
        "    out[f'st{int(dbl)}'] = m.stars\n"
        f"np.savez({str(tmp_path / 'w.npz')!r}, **out)\n")
    r = subprocess.run([sys.executable, "-c", script], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    z = np.load(tmp_path / "w.npz")
    for dbl in (False, True):
        m = irs_b200.IPM(**cfg, is_double=dbl)
        m.run()
        np.testing.assert_array_equal(z[f"mu{int(dbl)}"], m.magnifications)
        np.testing.assert_array_equal(z[f"st{int(dbl)}"], m.stars)
        m.close()


def _star_field(shape, rng):
    """A field that covers the starfile test lens's shooting region (kappa
    0.45, shear 0.4, light_loss 0.01, half length 2): equal masses, uniform
    in a disc of radius 56 (706 stars) or a rectangle of corner (11, 53) (167
    stars), i.e. kappa_star ~0.225."""
    if shape == "circle":
        n, rad = 706, 56.0
        r = rad * np.sqrt(rng.random(n))
        a = 2 * np.pi * rng.random(n)
        xy = np.stack([r * np.cos(a), r * np.sin(a)], 1)
        corner = (rad, 0.0)
    else:
        n, corner = 167, (11.0, 53.0)
        xy = (rng.random((n, 2)) * 2 - 1) * np.array(corner)
    return np.concatenate([xy, np.ones((n, 1))], 1), corner


@needs_ref
@pytest.mark.parametrize("fmt", ["txt", "bin_float", "bin_double"])
@pytest.mark.parametrize("shape", ["circle", "rect"])
def test_starfile_ingest_matches_reference(gpu, tmp_path, fmt, shape):
    """Star files (star.cuh:175-434): .txt (positions in units of the Einstein
    radius, the field's shape from its moment of inertia, theta 1) and .bin in
    float or double (told apart by the file size), through the reference's
    IPM and this build's on the same map: identical parameters, stars and maps
    (double builds)."""
    rng = np.random.default_rng(42)
    stars, corner = _star_field(shape, rng)
    if fmt == "txt":
        sf = str(tmp_path / "stars.txt")
        np.savetxt(sf, stars, fmt="%.17g")
    else:
        sf = str(tmp_path / "stars.bin")
        rg.write_starfile(sf, stars, shape == "rect", corner, 1.0, double=(fmt == "bin_double"))
    p = dict(kappa_tot=0.45, shear=0.4, light_loss=0.01, safety_scale=1.1, starfile=sf, half_length_y1=2.0,
             half_length_y2=2.0, num_pixels_y1=64, num_pixels_y2=64, num_rays_y=4, write_stars=1, write_maps=0,
             write_histograms=0)
    rd = tmp_path / "ref"
    rd.mkdir()
    r = rg.run_ipm(p, is_double=True, outdir=str(rd))
    m = irs_b200.IPM(**p, is_double=True, outfile_prefix=str(tmp_path / "ours_"))
    m.run()
    m.save()
    ours = rg.read_param_info(str(tmp_path / "ours_ipm_parameter_info.txt"))
    for k, v in r["param_info"].items():
        if k in SKIP_KEYS or isinstance(v, str):
            continue
        assert ours.get(k) == v, (k, ours.get(k), v)
    np.testing.assert_array_equal(_sorted(r["stars"]), _sorted(m.stars))
    med, p99, mx = rel_err(m.magnifications, r["magnifications"])
    assert med <= 1e-8 and p99 <= 1e-7, (med, p99, mx)
    m.close()


@needs_ref
def test_histograms_match_reference(gpu, tmp_path):
    """The histogram files (ipm.cuh:950-1120, array_functions.cuh:114-160,
    write_histogram :318-349): magnification x 1000 and log10 magnification x
    1000, rounded, as (value, count) pairs, from the same star field (double
    builds, whose maps agree to ~1e-10): the same bins, counts equal but for
    pixels whose value sits within rounding of a bin edge (at most 2 per bin)."""
    p = dict(headline_params(), half_length_y1=4.0, half_length_y2=4.0, num_pixels_y1=256, num_pixels_y2=256,
             write_stars=0, write_maps=0, write_histograms=1)
    rd = tmp_path / "ref"
    rd.mkdir()
    rg.run_ipm(p, is_double=True, outdir=str(rd))
    m = irs_b200.IPM(**p, is_double=True, outfile_prefix=str(tmp_path / "ours_"))
    m.run()
    m.save()
    for f in ("ipm_mags_numpixels.txt", "ipm_log_mags_numpixels.txt"):
        a = np.loadtxt(rd / f, dtype=np.int64).reshape(-1, 2)
        b = np.loadtxt(tmp_path / ("ours_" + f), dtype=np.int64).reshape(-1, 2)
        assert a[:, 1].sum() == b[:, 1].sum() == 256 * 256
        da, db = dict(map(tuple, a)), dict(map(tuple, b))
        for k in set(da) | set(db):
            assert abs(da.get(k, 0) - db.get(k, 0)) <= 2, (f, k, da.get(k), db.get(k))
        assert sum(abs(da.get(k, 0) - db.get(k, 0)) for k in set(da) | set(db)) <= 8, f
    m.close()
