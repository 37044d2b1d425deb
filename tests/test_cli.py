"""Command-line tools without a GPU: they exist after the build, and reject
wrong arguments and unreadable files with the reference tools' messages and
exit codes (cuxmss/ui/keypair.c, sign.c, open.c) before touching the GPU."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "cu-xmss_b200", "xmss_b200", "bin")
TOOLS = [p + k for p in ("xmss_", "xmssmt_") for k in ("keypair", "sign", "open")]


@pytest.mark.parametrize("tool", TOOLS)
def test_cli_usage(tool):
    exe = os.path.join(BIN, tool)
    assert os.access(exe, os.X_OK), f"{exe} not built (make -C cu-xmss_b200)"
    p = subprocess.run([exe], capture_output=True, timeout=60)
    assert p.returncode == 255 and p.stdout == b""
    assert p.stderr.startswith(b"Expected ")


@pytest.mark.parametrize("tool", ["xmss_sign", "xmss_open", "xmssmt_sign", "xmssmt_open"])
def test_cli_missing_files(tool, tmp_path):
    p = subprocess.run([os.path.join(BIN, tool), str(tmp_path / "nokey"), str(tmp_path / "nomsg")],
                       capture_output=True, timeout=60)
    assert p.returncode == 255 and p.stderr == b"Could not open keypair file.\n"


def test_cli_bad_params(tmp_path):
    p = subprocess.run([os.path.join(BIN, "xmss_keypair"), "XMSS-NOPE"], capture_output=True, timeout=60)
    assert p.returncode == 255 and p.stderr == b"Error parsing oid.\n"
