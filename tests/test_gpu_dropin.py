"""The reference's own test programs, unchanged, on libxmss_b200.so.

oracle/Makefile (`make -C oracle dropin`) compiles cuxmss/test/xmss.c (XMSS
and XMSS^MT, with and without XMSS_TEST_INVALIDSIG), test/xmss_determinism.c
and test/xmss_max_signatures.c from the reference's sources and headers and
links them against libxmss_b200.so alone, with a deterministic randombytes
(oracle/ref_randombytes.c) in place of /dev/urandom: none of the reference's
.c files is linked in.  Each program must exit 0 and print what the
reference's own run prints (cuxmss/test/xmss.c:39-144,
test/xmss_max_signatures.c:32-95).  The binaries are built where the
reference sources are present and travel with the repository.
"""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DROPIN = os.path.join(ROOT, "oracle", "_ref", "dropin")


def _run(prog, timeout=900):
    exe = os.path.join(DROPIN, prog)
    if not os.path.exists(exe):
        pytest.skip("built where the reference sources are present: make -C oracle dropin")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=timeout)
    out = r.stdout + r.stderr
    assert r.returncode == 0, f"{prog} exited {r.returncode}:\n{out[-3000:]}"
    return out


def test_binaries_link_only_the_library():
    exe = os.path.join(DROPIN, "xmss")
    if not os.path.exists(exe):
        pytest.skip("built where the reference sources are present: make -C oracle dropin")
    syms = subprocess.run(["nm", "-D", "--undefined-only", exe], capture_output=True, text=True).stdout
    assert "xmss_sign_open" in syms and "xmss_keypair" in syms  # resolved by the shared library
    need = subprocess.run(["readelf", "-d", exe], capture_output=True, text=True).stdout
    assert "libxmss_b200.so" in need and "libcrypto" not in need


@pytest.mark.parametrize("prog,sigs", [("xmss", 16), ("xmss_invalidsig", 16), ("xmssmt", 16),
                                       ("xmssmt_invalidsig", 16)])
def test_reference_xmss_program(prog, sigs):
    out = _run(prog)
    assert out.count("verification succeeded.") == sigs
    assert out.count("flipping a bit of m invalidates signature.") == sigs
    if "invalidsig" in prog:
        assert out.count("changing any signature hash invalidates signature.") == sigs
    assert "  X " not in out


def test_reference_determinism_program():
    out = _run("xmss_determinism")
    assert "signatures are identical." in out


def test_reference_max_signatures_program():
    """XMSS-SHA2_10_256: 1,024 signatures return 0 (the last with the wiped
    key), the next two return -2."""
    out = _run("xmss_max_signatures")
    assert "As expected, return code was 0" in out
    assert out.count("Return code as expected [-2].") == 2
