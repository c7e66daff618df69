"""The CPU oracle built with AddressSanitizer, UndefinedBehaviorSanitizer
and LeakSanitizer and driven through every entry point on small cases
(tests/cpp/oracle_sanitize.c): the checker of the device kernels must itself
be free of out-of-bounds accesses, leaks and undefined arithmetic."""
from __future__ import annotations

import os
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def test_oracle_is_clean_under_sanitizers(tmp_path):
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.fail("gcc not found")
    exe = tmp_path / "oracle_sanitize"
    srcs = sorted(str(p) for p in (ROOT / "oracle" / "src").glob("*.c"))
    cmd = [gcc, "-std=c11", "-O1", "-g", "-fsanitize=address,undefined", "-fno-sanitize-recover=all",
           "-fno-omit-frame-pointer", "-ffp-contract=off", *srcs, str(ROOT / "tests" / "cpp" / "oracle_sanitize.c"),
           "-lm", "-lpthread", "-o", str(exe)]
    out = subprocess.run(cmd, capture_output=True, text=True)
    assert out.returncode == 0, out.stderr[-4000:]
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=1:abort_on_error=0", UBSAN_OPTIONS="print_stacktrace=1")
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300, env=env)
    assert run.returncode == 0 and run.stdout.strip() == "ok", run.stderr[-4000:]
