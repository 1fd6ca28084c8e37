"""Command-line tools (the reference's ipm_gpu / irs_gpu interface)."""
import os
import subprocess

import numpy as np
import pytest

BIN = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "irs_b200", "bin")


def run(name, *args):
    return subprocess.run([os.path.join(BIN, name), *map(str, args)], capture_output=True, text=True, timeout=600)


@pytest.mark.parametrize("name", ["ipm_gpu", "ipm_gpu_double", "irs_gpu", "irs_gpu_double"])
def test_usage_and_syntax_errors(name):
    r = run(name, "-h")
    assert r.returncode == 255 and "--kappa_tot" in r.stdout and "--num_rays_y" in r.stdout
    r = run(name, "-k")
    assert r.returncode == 255 and "Invalid input syntax" in r.stderr
    r = run(name, "--nope", "1")
    assert r.returncode == 255 and "Unknown option --nope" in r.stderr
    r = run(name, "-k", "abc")
    assert r.returncode == 255 and "Invalid kappa_tot input" in r.stderr


@pytest.mark.gpu
def test_ipm_cli_writes_reference_files(gpu, tmp_path):
    pre = str(tmp_path) + "/"
    r = run("ipm_gpu", "-v", 0, "-k", 0.45, "-y", 0.4, "-s", 0.5, "-mf", "salpeter", "-ml", 0.08, "-mh", 1.0,
            "-t", 2.31, "-ll", 0.01, "-hly1", 4, "-hly2", 4, "-npy1", 128, "-npy2", 128, "-rs", 22, "-wp", 1,
            "-o", pre)
    assert r.returncode == 0, r.stderr
    info = dict(l.split() for l in open(tmp_path / "ipm_parameter_info.txt"))
    assert abs(float(info["kappa_star"]) - 0.225) < 1e-6
    a = np.fromfile(tmp_path / "ipm_magnifications.bin", dtype=np.int32, count=2)
    assert list(a) == [128, 128]
    mu = np.fromfile(tmp_path / "ipm_magnifications.bin", dtype=np.float32, offset=8).reshape(128, 128)
    mn = np.fromfile(tmp_path / "ipm_magnifications_minima.bin", dtype=np.float32, offset=8).reshape(128, 128)
    sd = np.fromfile(tmp_path / "ipm_magnifications_saddles.bin", dtype=np.float32, offset=8).reshape(128, 128)
    np.testing.assert_allclose(mu, mn + sd, rtol=1e-6)
    assert os.path.exists(tmp_path / "ipm_stars.bin")


@pytest.mark.gpu
def test_irs_cli_counts(gpu, tmp_path):
    pre = str(tmp_path) + "/"
    r = run("irs_gpu_double", "-v", 0, "-k", 0.4, "-y", 0.3, "-ks", 0.4, "-hly1", 3, "-hly2", 3, "-npy1", 96,
            "-npy2", 96, "-nry", 16, "-rs", 11, "-o", pre)
    assert r.returncode == 0, r.stderr
    info = dict(l.split() for l in open(tmp_path / "irs_parameter_info.txt"))
    counts = np.fromfile(tmp_path / "irs_magnifications.bin", dtype=np.int32, offset=8)
    assert counts.sum() == int(info["num_rays_received"])
    hist = np.loadtxt(tmp_path / "irs_numrays_numpixels.txt", dtype=np.int64)
    assert hist[:, 1].sum() == 96 * 96


@pytest.mark.parametrize("name,opt", [("ccf_gpu", "--num_phi"), ("ncc_gpu", "--over_sample")])
def test_ccf_ncc_usage_and_syntax_errors(name, opt):
    r = run(name, "-h")
    assert r.returncode == 255 and opt in r.stdout and "--outfile_prefix" in r.stdout
    r = run(name, "-v")
    assert r.returncode == 255 and "Invalid input syntax" in r.stderr
    r = run(name, "--nope", "1")
    assert r.returncode == 255 and "Unknown option --nope" in r.stderr
    r = run(name, "-v", "abc")
    assert r.returncode == 255 and "Invalid verbose input" in r.stderr


@pytest.mark.gpu
def test_ccf_then_ncc_cli(gpu, tmp_path):
    """ccf_gpu writes the critical curves and caustics; ncc_gpu maps the
    caustic crossings from ccf_caustics.bin, as the reference's tools do."""
    pre = str(tmp_path) + "/"
    r = run("ccf_gpu", "-v", 0, "-k", 0.3, "-y", 0.3, "-s", 0.1, "-ns", 40, "-np", 50, "-rs", 5, "-o", pre)
    assert r.returncode == 0, r.stderr
    info = dict(l.split() for l in open(tmp_path / "ccf_parameter_info.txt"))
    assert abs(float(info["kappa_star"]) - 0.27) < 1e-9 and info["num_roots"] == "80"
    assert float(info["max_error_1/mu"]) < 1e-8
    nr, nc = np.fromfile(tmp_path / "ccf_caustics.bin", dtype=np.int32, count=2)
    assert (nr, nc) == (80, 51)
    r = run("ncc_gpu", "-v", 0, "-ip", pre, "-hly1", 4, "-hly2", 4, "-npy1", 100, "-npy2", 100, "-os", 1, "-o", pre)
    assert r.returncode == 0, r.stderr
    m = np.fromfile(tmp_path / "ncc_ncc.bin", dtype=np.int32)
    assert list(m[:2]) == [100, 100] and m[2:].min() >= 0 and m[2:].max() >= 1
    assert os.path.exists(tmp_path / "ncc_ncc_numpixels.txt")
