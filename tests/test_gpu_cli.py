"""The command-line tools (cu-xmss_b200/cli/xmss_cli.c, built as
xmss[mt]_keypair / _sign / _open) against the reference's own ui/ programs
compiled from its sources into oracle/_ref/ui (oracle/Makefile): same
keypair files from the same randomness, same signature files, same in-place
key updates, each side verifying the other's signatures."""
import os
import shutil
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "cu-xmss_b200", "xmss_b200", "bin")
REF_UI = os.path.join(ROOT, "oracle", "_ref", "ui")


def run(exe, *args, cwd):
    p = subprocess.run([exe, *args], cwd=cwd, capture_output=True, timeout=300)
    return p.returncode, p.stdout


def det_keypair_tool(tmp, mt):
    """Our keypair tool linked with the reference tools' deterministic
    randombytes (the library's randombytes is interposable, as the
    reference's is)."""
    exe = os.path.join(tmp, "det_keypair" + ("_mt" if mt else ""))
    cmd = ["gcc", "-O2", "-DCLI_KEYPAIR"] + (["-DXMSSMT"] if mt else []) + [
        os.path.join(ROOT, "cu-xmss_b200", "cli", "xmss_cli.c"), os.path.join(ROOT, "oracle", "ref_randombytes.c"),
        "-I" + os.path.join(ROOT, "include"), "-L" + os.path.join(ROOT, "cu-xmss_b200", "xmss_b200"), "-lxmss_b200",
        "-Wl,-rpath," + os.path.join(ROOT, "cu-xmss_b200", "xmss_b200"), "-o", exe]
    subprocess.run(cmd, check=True)
    return exe


@pytest.mark.skipif(not os.path.isdir(REF_UI), reason="reference tools not built (oracle/Makefile ref)")
@pytest.mark.parametrize("mt,params", [(False, "XMSS-SHA2_10_256"), (True, "XMSSMT-SHA2_20/4_256")])
def test_cli_against_reference_tools(tmp_path, mt, params):
    t = str(tmp_path)
    pre = "xmssmt_" if mt else "xmss_"
    ours = {k: os.path.join(BIN, pre + k) for k in ("keypair", "sign", "open")}
    ref = {k: os.path.join(REF_UI, pre + k) for k in ("keypair", "sign", "open")}
    # keypair files: byte-identical from the same randomness
    rc, k_ref = run(ref["keypair"], params, cwd=t)
    assert rc == 0
    rc, k_ours = run(det_keypair_tool(t, mt), params, cwd=t)
    assert rc == 0 and k_ours == k_ref
    rng = np.random.default_rng(9)
    for i, mlen in enumerate((0, 33, 3000)):
        with open(os.path.join(t, "m"), "wb") as f:
            f.write(rng.bytes(mlen))
        for name in ("ka", "kb"):
            if i == 0:
                with open(os.path.join(t, name), "wb") as f:
                    f.write(k_ref)
        rc_a, sm_a = run(ours["sign"], "ka", "m", cwd=t)
        rc_b, sm_b = run(ref["sign"], "kb", "m", cwd=t)
        assert rc_a == rc_b == 0 and sm_a == sm_b, mlen
        assert open(os.path.join(t, "ka"), "rb").read() == open(os.path.join(t, "kb"), "rb").read()
        with open(os.path.join(t, "sm"), "wb") as f:
            f.write(sm_a)
        for tool in (ours["open"], ref["open"]):
            rc, out = run(tool, "ka", "sm", cwd=t)
            assert rc == 0 and out == b"Verification succeeded.\n"
        bad = bytearray(sm_a)
        bad[len(bad) // 2] ^= 0x04
        with open(os.path.join(t, "bad"), "wb") as f:
            f.write(bytes(bad))
        outs = [run(tool, "ka", "bad", cwd=t) for tool in (ours["open"], ref["open"])]
        assert outs[0] == outs[1] and outs[0][0] != 0 and outs[0][1] == b"Verification failed!\n"
    # our own keypair tool (system randomness): the reference verifies its signatures
    rc, k_new = run(ours["keypair"], params, cwd=t)
    assert rc == 0 and len(k_new) == len(k_ref) and k_new != k_ref
    with open(os.path.join(t, "kn"), "wb") as f:
        f.write(k_new)
    rc, sm = run(ours["sign"], "kn", "m", cwd=t)
    with open(os.path.join(t, "smn"), "wb") as f:
        f.write(sm)
    assert rc == 0 and run(ref["open"], "kn", "smn", cwd=t) == (0, b"Verification succeeded.\n")


@pytest.mark.skipif(not os.path.isdir(REF_UI), reason="reference tools not built (oracle/Makefile ref)")
def test_cli_last_index(tmp_path):
    """A keypair file at index 2^h - 1: both tools sign once with the wiped
    key (the reference's quirk, xmss_core.c:212-233: wiped, then index
    2^h stored) and write the same file; the next sign fails with -2 here
    (no signature) and both store the fully wiped key."""
    t = str(tmp_path)
    rc, k = run(os.path.join(REF_UI, "xmss_keypair"), "XMSS-SHA2_10_256", cwd=t)
    assert rc == 0
    k = bytearray(k)
    pk_len = 4 + 64
    k[pk_len + 4:pk_len + 8] = (1023).to_bytes(4, "big")
    for name in ("ka", "kb"):
        with open(os.path.join(t, name), "wb") as f:
            f.write(bytes(k))
    with open(os.path.join(t, "m"), "wb") as f:
        f.write(b"last")
    rc_a, sm_a = run(os.path.join(BIN, "xmss_sign"), "ka", "m", cwd=t)
    rc_b, sm_b = run(os.path.join(REF_UI, "xmss_sign"), "kb", "m", cwd=t)
    assert rc_a == rc_b == 0 and sm_a == sm_b
    ka = open(os.path.join(t, "ka"), "rb").read()
    assert ka == open(os.path.join(t, "kb"), "rb").read()
    assert ka[pk_len + 4:pk_len + 8] == (1024).to_bytes(4, "big") and ka[pk_len + 8:] == bytes(len(ka) - pk_len - 8)
    rc, sm = run(os.path.join(BIN, "xmss_sign"), "ka", "m", cwd=t)
    assert rc == 256 - 2 and sm == b""
    run(os.path.join(REF_UI, "xmss_sign"), "kb", "m", cwd=t)  # returns 0 and prints an unset buffer
    ka = open(os.path.join(t, "ka"), "rb").read()
    assert ka == open(os.path.join(t, "kb"), "rb").read()
    assert ka[pk_len + 4:pk_len + 8] == b"\xff" * 4
