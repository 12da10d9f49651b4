"""Host-side pieces of bench.py that need no GPU: the reference's run over a
pixel window (the CPU baselines of the batch, guiding and large-scene
sections) and the committed ncu traffic summaries that the rooflines scale."""
import importlib.util
import json
import os

import pytest

from conftest import ROOT


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_reference_window_renders_exactly_the_window(oracle, scenes):
    """The harness's profiler area (cpuMulticore.cu:17) renders the window's
    pixels at the requested spp and nothing else."""
    if not oracle.ref_available():
        pytest.skip("oracle/_ref/cr_ref not built")
    bench = _bench()
    d = scenes.config0()
    samples, seconds, threads = bench.reference_window(d, 2, 7, (100, 96, 132, 120))
    assert samples == 32 * 24 * 2
    assert seconds > 0 and threads >= 1
    full, _, _ = bench.reference_window(d, 1, 7)
    assert full == d.width * d.height


@pytest.mark.parametrize("name, key", [("k_extend_traffic.json", "dram_bytes_per_ray"),
                                       ("k_extend_traffic_config4.json", "dram_bytes_per_ray"),
                                       ("k_guide_infer_traffic.json", "dram_bytes_per_row")])
def test_traffic_summaries_carry_what_the_rooflines_read(name, key):
    bench = _bench()
    t = bench.profiled_traffic(name)
    assert t is not None, name
    assert t[key] > 0
    assert t["dram_bytes_read"] + t["dram_bytes_write"] > 0
    assert "ncu" in t["command"] and "--clock-control none" in t["command"]
    with open(os.path.join(ROOT, "profiles", name)) as fh:
        assert json.load(fh) == t
