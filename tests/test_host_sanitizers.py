"""Host code under AddressSanitizer / UndefinedBehaviorSanitizer (no GPU):
the dependency-level schedule builder of the fused sweep
(ccd_b200/csrc/schedule.cpp) with a fuzz test of its invariants, the
multi-threaded row-major copy (ccd_b200/csrc/csr_host.cpp) against a plain
counting sort (also under ThreadSanitizer), and the oracle restatement
(oracle/ccd_oracle.c) through every call on random problems.  compute-sanitizer is not used for the device side; these cover the
host side the way the reference's ASAN/UBSAN builds cover its C++."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SAN = ["-O1", "-g", "-fsanitize=address,undefined", "-fno-sanitize-recover=all", "-fno-omit-frame-pointer"]

pytestmark = pytest.mark.skipif(shutil.which("g++") is None or shutil.which("gcc") is None,
                                reason="no host compiler")


def _build_and_run(cmd, exe, args, timeout=600):
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]
    r = subprocess.run([exe] + args, capture_output=True, text=True, timeout=timeout)
    assert r.returncode == 0, (r.stdout[-2000:], r.stderr[-6000:])
    return r.stdout


@pytest.mark.timeout(900)
def test_schedule_builder_fuzz_under_sanitizers(tmp_path):
    exe = str(tmp_path / "schedule_check")
    out = _build_and_run(["g++", "-std=c++17"] + SAN + ["-I" + os.path.join(ROOT, "ccd_b200", "csrc"),
                          os.path.join(ROOT, "tests", "native", "schedule_check.cpp"),
                          os.path.join(ROOT, "ccd_b200", "csrc", "schedule.cpp"), "-o", exe], exe, ["400"])
    assert "schedules checked" in out


@pytest.mark.timeout(900)
def test_oracle_under_sanitizers(tmp_path):
    exe = str(tmp_path / "oracle_check")
    out = _build_and_run(["gcc", "-std=c11"] + SAN + ["-I" + os.path.join(ROOT, "oracle"),
                          os.path.join(ROOT, "tests", "native", "oracle_check.c"),
                          os.path.join(ROOT, "oracle", "ccd_oracle.c"), "-lm", "-o", exe], exe, ["200"])
    assert "ran clean" in out


@pytest.mark.timeout(900)
@pytest.mark.parametrize("sanitizer", [SAN, ["-O1", "-g", "-fsanitize=thread"]], ids=["asan_ubsan", "tsan"])
def test_row_major_copy_under_sanitizers(tmp_path, sanitizer):
    exe = str(tmp_path / "csr_check")
    csrc = os.path.join(ROOT, "ccd_b200", "csrc")
    out = _build_and_run(["g++", "-std=c++17"] + sanitizer + ["-I" + csrc,
                          os.path.join(ROOT, "tests", "native", "csr_check.cpp"),
                          os.path.join(csrc, "csr_host.cpp"), "-lpthread", "-o", exe], exe, ["100"])
    assert "identical" in out
