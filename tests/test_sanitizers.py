"""The library's host code (setup, quadrature, samplers, worker pool, the
host side of the device-assisted sampler) and the C oracle built with
AddressSanitizer and UndefinedBehaviorSanitizer and run on the CPU: any
report aborts the driver (tests/sanitize_driver.cpp), which also checks setup
and tables against the oracle, and the device-assisted sampler against the
serial one, bit for bit. The CUDA runtime and the sampler kernels are
emulated on the host inside the driver; no GPU is reached."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
CSRC = ROOT / "scarf3d_b200" / "csrc"
CUDA = Path("/usr/local/cuda")
SAN = ["-fsanitize=address,undefined", "-fno-sanitize-recover=all", "-fno-omit-frame-pointer", "-g", "-O1",
       "-ffp-contract=off"]


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    if not shutil.which("g++") or not (CUDA / "include" / "cuda_runtime.h").exists():
        pytest.skip("g++ or CUDA headers missing")
    d = tmp_path_factory.mktemp("san")
    orc = d / "srm_oracle.o"
    subprocess.run(["gcc", "-std=c11", *SAN, "-c", str(ROOT / "oracle" / "srm_oracle.c"), "-o", str(orc)],
                   check=True)
    exe = d / "sanitize_driver"
    subprocess.run(["g++", "-std=c++17", *SAN, f"-I{ROOT / 'include'}", f"-I{CSRC}", f"-I{CUDA / 'include'}",
                    str(Path(__file__).with_name("sanitize_driver.cpp")), str(CSRC / "srm_host.cpp"),
                    str(CSRC / "srm_quad.cpp"), str(orc), "-lpthread", "-lm", "-o", str(exe)], check=True)
    return exe


def test_host_code_is_clean_under_asan_and_ubsan(driver):
    r = subprocess.run([str(driver)], capture_output=True, text=True, timeout=600,
                       env={"ASAN_OPTIONS": "detect_leaks=0", "UBSAN_OPTIONS": "print_stacktrace=1",
                            "PATH": "/usr/bin:/bin"})
    assert r.returncode == 0, r.stdout + r.stderr
    assert "5 cases, 21 device-sampler batches, 0 failures" in r.stdout
