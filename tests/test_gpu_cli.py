"""The sj_main command line (the reference's main.cu interface) on a B200.

Runs the CLI on a CSV the way the reference's binary is run (`<dataset.csv>
<epsilon> <ndim> <searchmode>`), with --print, and checks every printed
neighbour list against the oracle on the same imported points (the CLI imports
with the reference's parse and bin sort, so ids are those of sjoin.read_csv),
the printed result-set size, and the stats line appended to the per-mode file
of main.cu:88-150 / 203-206.
"""
import os
import re
import subprocess

import numpy as np
import pytest

import oracle
import sjoin
from conftest import PKG_DIR, exp_points

pytestmark = pytest.mark.gpu

CLI = os.path.join(PKG_DIR, "sjoin", "sj_main")
STATS = {3: "gpu_global_stats.txt", 5: "gpu_b-unicomp_stats.txt", 8: "gpu_dynamic-threads-fixed_stats.txt",
         10: "gpu_working-queue_lid-unicomp_stats.txt"}


@pytest.mark.parametrize("mode", [3, 5, 8, 10])
def test_cli_prints_the_oracle_neighbour_lists(tmp_path, mode):
    pts = exp_points(3000, 2, 11)
    eps = 0.004
    csv = tmp_path / "data.csv"
    sjoin.datasets.write_csv(str(csv), pts)
    out = subprocess.run([CLI, str(csv), repr(eps), "2", str(mode), "--print"], cwd=tmp_path, capture_output=True,
                         text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    imported = sjoin.read_csv(str(csv), 2)
    keys, vals = oracle.OracleIndex(imported, eps, 2).pairs()
    deg = np.bincount(keys, minlength=len(imported))
    total = int(re.search(r"Total result set size: (\d+)", out.stdout).group(1))
    assert total == len(keys)
    rows = re.findall(r"point id: (\d+), neighbors: nb neighbor (\d+)\n([0-9,]*)", out.stdout)
    assert len(rows) == len(imported)
    start = np.concatenate([[0], np.cumsum(deg)])
    for pid, nb, lst in rows:
        i = int(pid)
        got = [int(x) for x in lst.split(",") if x]
        assert int(nb) == deg[i] == len(got)
        assert got == sorted(vals[start[i]:start[i + 1]].tolist())
    line = open(tmp_path / STATS[mode]).read().strip().splitlines()[-1]
    parts = [x.strip() for x in line.split(",")]
    assert parts[1] == str(csv) and int(parts[3]) == len(keys)
    assert "GPUNUMDIM/NUMINDEXEDDIM/DTYPE/BLOCKSIZE/THperPOINT/SORT: 2" in line
