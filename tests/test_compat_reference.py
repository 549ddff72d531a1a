"""Drop-in proof: the reference's own test programs (tests/*.cpp|cu of
nikitaborisov/birdwing), compiled unmodified against this repository's
compatible headers (include/) and linked with libbirdwing, in all three
limb-width configurations; beside them the reference's own host code and
stage kernels run under its own tests.  Built by oracle/build_ref.sh into
oracle/_ref/ (needs the reference tree; skipped when not built)."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref")
WIDTHS = ["32", "hybrid", "native"]
FAIL = re.compile(r"FAIL|MISMATCH|Mismatch|mismatch")


def run_bin(kind, width, name, tmp_path, timeout=600):
    path = os.path.join(REF, f"{kind}_{width}", name)
    if not os.path.exists(path):
        pytest.skip(f"{path} not built (oracle/build_ref.sh needs the reference tree)")
    p = subprocess.run([path], cwd=tmp_path, capture_output=True, text=True, timeout=timeout)
    out = p.stdout + p.stderr
    return p.returncode, out


def assert_passed(rc, out, min_pass=1):
    assert rc == 0, out[-3000:]
    bad = [ln for ln in out.splitlines() if FAIL.search(ln) and "0 failed" not in ln]
    assert not bad, "\n".join(bad[:20])
    assert len(re.findall(r"PASS|MATCH|OK", out)) >= min_pass, out[-2000:]


@pytest.mark.parametrize("kind", ["ref", "compat"])
@pytest.mark.parametrize("width", WIDTHS)
@pytest.mark.parametrize("name", ["test_crt", "test_ntt_limits"])
def test_host_programs(kind, width, name, tmp_path):
    rc, out = run_bin(kind, width, name, tmp_path)
    assert_passed(rc, out, 3)


@pytest.mark.gpu
@pytest.mark.parametrize("width", WIDTHS)
@pytest.mark.parametrize("name", ["test_zero_pad", "test_crt_gpu", "test_carry_prop"])
def test_reference_stage_kernels(width, name, tmp_path):
    """The reference's stage kernels under the reference's tests (baseline)."""
    rc, out = run_bin("ref", width, name, tmp_path)
    assert_passed(rc, out)


@pytest.mark.gpu
@pytest.mark.parametrize("width", WIDTHS)
@pytest.mark.parametrize("name", ["test_zero_pad", "test_crt_gpu", "test_carry_prop",
                                  "test_gpu_ntt_smoke", "test_pointwise_mul"])
def test_compat_stage_programs(width, name, tmp_path):
    """The reference's tests against this repository's stage kernels and
    lifecycle shims."""
    rc, out = run_bin("compat", width, name, tmp_path)
    assert_passed(rc, out, 0 if name == "test_pointwise_mul" else 1)


@pytest.mark.gpu
@pytest.mark.parametrize("width", WIDTHS)
def test_compat_full_multiply(width, tmp_path):
    """tests/test_full_multiply.cpp (schoolbook and GMP checks, sizes up to
    2^22 limbs) against host_multiply_merge / _native over libbirdwing."""
    rc, out = run_bin("compat", width, "test_full_multiply", tmp_path, timeout=1200)
    assert_passed(rc, out, 5)
