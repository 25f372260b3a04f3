"""CPU: the oracle restatement under AddressSanitizer and
UndefinedBehaviorSanitizer (every report fatal), over all its entry points
(tests/oracle_sanitized_battery.py)."""
import os
import shutil
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ASAN_SO = os.path.join(ROOT, "oracle", "_build", "liboracle_asan.so")


def _runtime(cc, name):
    p = subprocess.run([cc, f"-print-file-name={name}"], capture_output=True, text=True).stdout.strip()
    return p if os.path.isabs(p) and os.path.exists(p) else None


def test_oracle_battery_under_sanitizers():
    cc = shutil.which("gcc")
    asan = cc and _runtime(cc, "libasan.so")
    ubsan = cc and _runtime(cc, "libubsan.so")
    if not (asan and ubsan):
        pytest.skip("gcc sanitizer runtimes not available")
    subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "port-asan", f"SAN_CC={cc}"],
                   check=True, capture_output=True)
    env = dict(os.environ, PLSPARSE_ORACLE_LIB=ASAN_SO, LD_PRELOAD=f"{asan}:{ubsan}",
               ASAN_OPTIONS="detect_leaks=0:abort_on_error=0:exitcode=23",
               UBSAN_OPTIONS="halt_on_error=1:print_stacktrace=1:exitcode=24")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "tests", "oracle_sanitized_battery.py")],
                       env=env, capture_output=True, text=True, timeout=600)
    out = r.stdout + r.stderr
    assert r.returncode == 0, out[-4000:]
    assert "oracle battery ok" in r.stdout
    assert "AddressSanitizer" not in out and "runtime error" not in out, out[-4000:]
