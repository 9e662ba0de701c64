"""Target-sharded stepping of one system (pawan_b200.shard): the exchange
choreography on gloo ranks on the CPU, and the partition.  The GPU side
(pgpu_set_target_range / pgpu_stage / pgpu_records) is tested on one GPU in
test_shard_gpu.py."""
import os
import socket
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O
from pawan_b200 import cases
from pawan_b200.shard import partition

HERE = Path(__file__).resolve().parent


def test_partition_covers_every_target_once():
    for n in (0, 1, 7, 400, 425, 1001):
        for world in (1, 2, 3, 8):
            got = [partition(n, world, r) for r in range(world)]
            covered = np.zeros(n, int)
            for f, c, chunk in got:
                assert 0 <= c <= chunk
                covered[f:f + c] += 1
            assert np.all(covered == 1)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_match_single_process_rk4(tmp_path, world):
    """world ranks (425 particles: ragged blocks for 2 and 3 ranks) step two
    RK4 steps, exchanging the owned source records after every stage; the
    gathered state equals PAWAN's RK4 restated on one process, and the
    diagnostics combined from the ranks' fields (pgpu_diagnose_combine after
    an all-reduce) equal the restated diagnose of that state."""
    out = tmp_path / "state.npz"
    env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(_free_port()), WORLD_SIZE=str(world),
               STATIONS="17", OMP_NUM_THREADS="1")
    procs = [subprocess.Popen([sys.executable, str(HERE / "shard_worker.py"), str(out)], env=dict(env, RANK=str(r)))
             for r in range(world)]
    try:
        codes = [p.wait(timeout=180) for p in procs]
    finally:
        for p in procs:
            if p.poll() is None:
                p.kill()
    assert codes == [0] * world
    got = np.load(out)
    w = cases.ring_stations(stations=17, seed=0)
    pos, alpha = O.restate_step(w, 1e-4, "rk4", 0.01, 2)
    assert O.rel_err(got["pos"] - w.pos, pos - w.pos) < 1e-12
    assert O.rel_err(got["alpha"], alpha) < 1e-12
    ref, vbi = O.restate_diagnose(cases.Wake(got["pos"], got["alpha"], w.sigma, w.vol))
    scale = abs(ref[12])
    assert np.all(np.abs(got["diag"] - ref) <= 1e-12 * np.maximum(np.abs(ref), scale))
    assert np.all(np.abs(got["vbi"] - vbi) <= 1e-12 * np.abs(vbi).max())
