"""The whole program on the GPU (config.json -> TaskLyapunov over the C ABI
-> Data/Lyapunov shimizu.json) against the reference program's own output
file for the same config (tests/golden/program_*): identical bytes, for the
FD, VAR and QR methods."""
import os
import shutil
import subprocess

import pytest

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("method", ["fd", "var", "qr"])
def test_program_output_identical_to_reference(lib, tmp_path, method):
    cli = os.path.join(os.path.dirname(lib.LIB_PATH), "chaos_lyapunov")
    assert os.path.exists(cli), "command-line program not built"
    shutil.copy(os.path.join(GOLDEN, f"program_{method}_config.json"), tmp_path / "config.json")
    (tmp_path / "Data").mkdir()
    r = subprocess.run([cli, "--model", "shimizu"], cwd=tmp_path, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    got = (tmp_path / "Data" / "Lyapunov shimizu.json").read_bytes()
    want = open(os.path.join(GOLDEN, f"program_{method}_output.json"), "rb").read()
    assert got == want
