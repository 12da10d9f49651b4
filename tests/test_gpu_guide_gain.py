"""What the trained guide gains over the method without it: on the occluded-
light scene of the guiding benchmark (light behind a wall with a small
aperture, Beckmann receivers of roughness 0.05-0.5), after online training
the guided MIS estimator reaches a clearly lower relMSE than plain MIS at the
same number of samples per pixel."""
import numpy as np
import pytest

from conftest import require_gpu

pytestmark = pytest.mark.gpu

RES = 256


def _film(torch):
    n = RES * RES
    return [torch.zeros(n * 3, dtype=torch.float64, device="cuda"), torch.zeros(n * 3, dtype=torch.float64, device="cuda"),
            torch.zeros(n, dtype=torch.int32, device="cuda")]


def test_trained_guide_lowers_error_at_equal_spp(cr, scenes):
    require_gpu()
    import torch
    sc = cr.Scene.from_desc(scenes.config3(level=6, width=RES, height=RES))
    stream = torch.cuda.current_stream().cuda_stream

    def render(f, spp, seed, guiding, wave=0):
        d = cr.render_desc(RES, RES, spp, max_bounce=7, estimator=cr.MIS, seed=seed, guiding=guiding, wave_paths=wave)
        sc.render_device(d, f[0].data_ptr(), f[1].data_ptr(), f[2].data_ptr(), stream=stream, stats=False)

    # reference: plain MIS at 8192 spp
    R = _film(torch)
    for i in range(64):
        render(R, 128, 10_000 + i, False)
    c = R[2].double().repeat_interleave(3)
    Rm = R[0] / c
    Rvar = (R[1] / c - Rm * Rm).clamp_min(0) / c
    den = Rm * Rm + 1e-2

    def relmse(f):
        cc = f[2].double().repeat_interleave(3)
        return ((((f[0] / cc) - Rm) ** 2 - Rvar) / den).mean().item()

    # online training on the tracer's own paths (guided renders train as they go)
    g = cr.Guide(sc).reset(seed=5)
    g.configure(steps_per_wave=16, max_steps=600)
    T = _film(torch)
    for i in range(32):
        render(T, 16, 500 + i, True, wave=1 << 18)
    assert g.info()["step"] == 600  # trained to its budget, then frozen
    plain, guided = [], []
    for rep in range(4):
        for guiding, out in ((False, plain), (True, guided)):
            F = _film(torch)
            render(F, 256, 90_000 + 10 * rep + int(guiding), guiding)
            out.append(relmse(F))
    ratio = np.mean(guided) / np.mean(plain)
    print(f"GUIDE GAIN relMSE at 256 spp: plain {np.mean(plain):.3e} guided {np.mean(guided):.3e} ratio {ratio:.3f}")
    assert ratio < 0.85, (plain, guided)
