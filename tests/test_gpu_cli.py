"""The `cr` command line end to end on the GPU (src/cr.cu:9-68 drop-in)."""
import os
import subprocess

import numpy as np
import pytest

from conftest import require_gpu

pytestmark = pytest.mark.gpu


def test_cli_renders_png_and_pfm(cr, scenes, tmp_path):
    require_gpu()
    d = scenes.config0()
    path = scenes.write_scene(d, str(tmp_path), fmt="obj")
    out, pfm = str(tmp_path / "a.png"), str(tmp_path / "a.pfm")
    r = subprocess.run([cr.CLI_PATH, path, "-s", "4", "--resolution=40x30", "-o", out, "--pfm", pfm,
                        "-k", "Radiance"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert open(out, "rb").read(8) == b"\x89PNG\r\n\x1a\n"
    with open(pfm, "rb") as fh:
        head = fh.readline() + fh.readline() + fh.readline()
        img = np.frombuffer(fh.read(), "<f4").reshape(30, 40, 3)
    assert head.startswith(b"PF") and np.isfinite(img).all() and img.mean() > 0.05
    # the reference's debug kernels are selected the same way; unknown names fail
    nrm = str(tmp_path / "n.pfm")
    r = subprocess.run([cr.CLI_PATH, path, "-s", "2", "--resolution=40x30", "-o", out, "--pfm", nrm, "-k", "Normal"],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    with open(nrm, "rb") as fh:
        fh.readline(), fh.readline(), fh.readline()
        img = np.frombuffer(fh.read(), "<f4").reshape(30, 40, 3)
    assert np.isfinite(img).all() and 0.0 <= img.min() and img.max() <= 1.0  # n * 0.5 + 0.5
    bad = subprocess.run([cr.CLI_PATH, path, "-k", "Bogus", "-o", out], capture_output=True, text=True)
    assert bad.returncode != 0 and "not registered" in bad.stderr
