"""The C++ host path: pmp_spray_driver drives the update through
pmp::SprayParticleContainer (the C++ mirror of the reference container) with
host views, as a PeleLMeX time step would (moveKickDrift + moveKick per step).
Its droplets must equal the oracle's bit for bit, its summed deposits within
1e-12 of the largest; errors surface as the reference's abort messages."""
import os
import subprocess

import numpy as np
import pytest

from pelemp_b200 import build, workloads as W
from pelemp_b200.problem_io import read_result, write_problem
from tests.gpu_util import assert_bitwise, oracle_run
from tests.parity import source_errors

pytestmark = pytest.mark.gpu


def _driver():
    build.build_lib()
    return build.build_driver()


def test_cpp_driver_matches_oracle(tmp_path, oracle):
    prob = W.config2(n=20_000, steps=2, ncells=(32, 32, 32), box=(16, 16, 16))
    write_problem(prob, str(tmp_path))
    out = subprocess.run([_driver(), str(tmp_path)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    assert "ok substeps=" in out.stdout
    parts, srcs = read_result(prob, str(tmp_path))
    po, so = oracle_run(oracle, prob, prob.steps)
    assert_bitwise(parts, po)
    total = [sum(call[b] for call in so) for b in range(len(prob.boxes))]
    assert source_errors(total, srcs) <= 1e-12


def test_cpp_driver_reports_reference_abort(tmp_path):
    prob = W.walls(n=300, steps=1)
    prob.parts[0]["pos"][2, 4] = -0.5 * prob.dx[2]
    write_problem(prob, str(tmp_path))
    out = subprocess.run([_driver(), str(tmp_path)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 11
    assert "Particle has incorrectly left the domain" in out.stderr
    assert "droplet 4" in out.stderr
