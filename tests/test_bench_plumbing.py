"""bench.py plumbing on the CPU: the multi-rank timing reduction over gloo
(world size 2, one process per rank, as torchrun launches them) and the JSON
line of the `--impl reference` arm on a small workload."""
import json
import os
import socket
import subprocess
import sys

import pytest

from conftest import REPO


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


WORKER = r"""
import os, sys
sys.path.insert(0, {repo!r})
import bench
rank, local, world = bench.dist_env()
dist = bench.init_dist(world, "gloo")
bench.barrier(dist)
t = bench.max_over_ranks(10.0 + 5.0 * rank, dist)
print("RESULT", rank, t, flush=True)
dist.destroy_process_group()
"""


def test_max_over_ranks_with_gloo_two_ranks():
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, "-c", WORKER.format(repo=REPO)], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True))
    outs = [p.communicate(timeout=120)[0] for p in procs]
    for p, o in zip(procs, outs):
        assert p.returncode == 0, o
    vals = sorted(float(line.split()[2]) for o in outs for line in o.splitlines() if line.startswith("RESULT"))
    assert vals == [15.0, 15.0]


def test_reference_arm_prints_contract_line():
    cmd = [sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference", "--workload", "cornell_small",
           "--steps", "1", "--warmup", "0"]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=REPO)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads([l for l in out.stdout.splitlines() if l.startswith("{")][-1])
    assert line["impl"] == "reference"
    assert line["unit"] == "Msamples/s" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] in ("reference", "port")
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["value"] == line["value"]
    # a step is the sample itself, timed whole: 32 centre rows x 256 px x 8 spp
    assert "timed in full" in line["cpu_baseline"]["sample"]
    assert abs(line["value"] - 32 * 256 * 8 / (line["ms_per_step"] / 1e3) / 1e6) < 1e-6 * line["value"]


def test_reference_arm_other_ranks_exit_quietly():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2")
    out = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference", "--steps", "1"],
                         capture_output=True, text=True, timeout=120, cwd=REPO, env=env)
    assert out.returncode == 0 and out.stdout.strip() == ""


def test_profile_fields_parsed():
    """The roofline's traffic and limiter come from the committed ncu
    summary of the dominant kernel."""
    sys.path.insert(0, REPO)
    import bench
    prof = bench.read_profile("wf_trace", "export_frame")
    assert prof["traffic_bytes_per_launch"] > 0 and prof["bound"] == "issue"
    assert 0 < prof["simt_efficiency"] <= 32 and 0 < prof["issue_active"] <= 1


def test_algorithmic_bytes_units():
    sys.path.insert(0, REPO)
    import bench
    ctr = {k: 0 for k in ("node_tests", "tri_tests", "surface_hits", "light_samples", "closest_rays",
                          "shadow_rays", "photon_node_tests", "photon_tri_tests")}
    ctr.update(node_tests=10, tri_tests=2, closest_rays=3, shadow_rays=1)
    assert bench.algorithmic_bytes("wf_trace", ctr, 0) == 10 * 32 + 2 * 36
    assert bench.state_bytes("wf_trace", ctr) == 3 * 48 + 80
    ctr.update(surface_hits=4, light_samples=2)
    assert bench.algorithmic_bytes("render", ctr, 5) == 10 * 32 + 2 * 36 + 4 * 104 + 2 * 80 + 5 * 20
