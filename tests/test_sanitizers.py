"""The host analysis and the plan file round trip, built with the
compiler's sanitizers around a small driver
(tests/sanitize/analysis_driver.cpp), run clean: no data race under
ThreadSanitizer in the threaded steps, no out-of-bounds access or undefined
behaviour under AddressSanitizer + UBSan.  Skipped where the compiler has
no sanitizer runtime."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "recblock-sptrsv_b200", "csrc")


@pytest.mark.parametrize("flags", [["-fsanitize=thread"],
                                   ["-fsanitize=address,undefined", "-fno-sanitize-recover=undefined"]],
                         ids=["thread", "address+undefined"])
def test_host_analysis_under_sanitizer(tmp_path, flags):
    cxx = shutil.which("g++")
    if not cxx:
        pytest.skip("no g++")
    exe = str(tmp_path / "driver")
    build = subprocess.run([cxx, "-O1", "-g", "-std=c++17", "-pthread", *flags,
                            "-I" + os.path.join(ROOT, "include"), "-I" + CSRC, "-I/usr/local/cuda/include",
                            os.path.join(ROOT, "tests", "sanitize", "analysis_driver.cpp"),
                            os.path.join(CSRC, "analysis.cpp"), os.path.join(CSRC, "plan_io.cpp"), "-o", exe],
                           capture_output=True, text=True)
    if build.returncode != 0:
        if "cannot find" in build.stderr and "san" in build.stderr:
            pytest.skip("no sanitizer runtime")
        pytest.fail(build.stderr[-2000:])
    env = dict(os.environ, RBS_HOST_THREADS="8", TSAN_OPTIONS="halt_on_error=1", ASAN_OPTIONS="detect_leaks=1")
    run = subprocess.run([exe, str(tmp_path / "plan.rbs")], capture_output=True, text=True, env=env, timeout=900)
    out = run.stdout + run.stderr
    assert run.returncode == 0 and "analysis driver: ok" in out, out[-4000:]
    assert "Sanitizer" not in out and "runtime error" not in out, out[-4000:]
