"""Host-side logic of the request loop, on the CPU: the device-range allocator
that admission by device footprint rests on (compiled with g++ and run), and the
C ABI's argument checks that need no GPU."""
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def test_range_arena(tmp_path):
    exe = tmp_path / "arena_check"
    subprocess.run(["g++", "-O1", "-std=c++17", "-o", str(exe), os.path.join(HERE, "cpp", "arena_check.cpp")],
                   check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0 and out.stdout.strip() == "ok", out.stdout


def test_server_create_without_gpu_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from hpc_ode_b200 import native
    with pytest.raises(native.B200Error) as e:
        native.Server()
    assert e.value.code == 5   # B200ODE_ERR_NO_DEVICE
