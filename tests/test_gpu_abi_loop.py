"""KORAL's RK2 time loop (ko.c:571-626) written in C against the C-ABI,
operator by operator (begin_step, save_timesteps, copyi_u, do_correct,
op_explicit, calc_u2p, op_implicit, addi_u into the k2 array ut2), gives
the same bytes as the fused device step kgpu_rk2_steps: on the Orszag-Tang
vortex and on the magnetised Kerr torus with its boundaries and floors."""
import subprocess

import pytest

from test_abi import build_rk2_loop

pytestmark = pytest.mark.gpu


def test_per_operator_loop_bit_identical_to_fused_step(kgpu, tmp_path):
    exe = build_rk2_loop(kgpu, tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    print(r.stdout, r.stderr)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.count("bit-identical") == 2
