"""The bench's reference arm without a CUDA device: it falls back to the
FP32 host C++/OpenMP restatement of the reference operators (kind "port")
and prints one JSON line with the fields the harness reads."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_falls_back_to_the_host_port():
    env = {**os.environ, "CUDA_VISIBLE_DEVICES": ""}
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "1"], cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["metric"] == "slots/s" and d["value"] > 0
    assert d["higher_is_better"] is True
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert d["config"]["iq_dtype"] == "int8" and d["config"]["workload"].startswith("uplink slot 256x32")


def test_reference_arm_maps_none_of_this_projects_libraries():
    """The reference arm's process loads the slot generator from its file and
    never imports the package, so libmegastation_b200.so is not mapped."""
    code = ("import sys; sys.argv=['bench.py']; import bench; d = bench._standalone_datagen(); "
            "c = d.CellConfig(M=8, K=4, N=64, S=48, U=1, iq_dtype='int8'); s = d.make_slot(c); "
            "assert s['iq'].dtype.name == 'int8'; "
            "assert 'megastation_b200' not in sys.modules, 'package imported'; "
            "maps = open('/proc/self/maps').read(); "
            "assert 'libmegastation_b200' not in maps, 'library mapped'; print('ok')")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "ok" in r.stdout, r.stderr[-2000:]


def test_generator_helpers_match_the_library():
    """The generator's numpy LDPC sizing and pilot values agree with the
    library's host functions (mb_ldpc_sizes, mb_pilot_sign)."""
    import numpy as np

    from megastation_b200 import datagen, ops
    for S in (16, 192, 600, 1200, 3276, 4000):
        for Qm in (2, 4, 6, 8):
            for rate in (1 / 3, 0.5, 0.8):
                for bg in (1, 2):
                    assert tuple(datagen.ldpc_sizes(S, Qm, rate, bg)) == tuple(ops.ldpc_sizes(S, Qm, rate, bg))
        ps = ops.pilot_sign(S).numpy()
        assert np.abs(datagen.pilot_values(S) - ps / np.abs(ps) ** 2).max() < 1e-6
