"""The boundary from C and C++: include/sparkit_b200.h compiled as strict
C99 against the library, and the C++ drop-in include/sparkit_b200.hpp
compiled with the sparkit reference's own headers (tests/cpp/build.sh).

Without a GPU: the C99 program runs, the drop-in reports SK_NO_DEVICE from
its constructor, and the two misuses (a host lambda given to a device
overload, a device operator given to a reference solver) fail to compile
with the library's message.  On a B200 the drop-in runs the configuration-1
Jacobi-CG, BiCGSTAB, FGMRES(30) and the four product formats next to the
reference's own solvers and multiply, with the same config structs
(tests/cpp/dropin_test.cpp)."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CPP = os.path.join(ROOT, "tests", "cpp")
BUILD = os.path.join(CPP, "_build")
REF = "/root/reference"


def _build():
    subprocess.run(["bash", os.path.join(CPP, "build.sh")], check=True, capture_output=True, timeout=600)


def _ref_available():
    return os.path.isfile(os.path.join(REF, "sparkit", "config.hpp.in")) and os.path.isfile(
        os.path.join(ROOT, "oracle", "_ref", "libsparkit_ref.so"))


def test_c_header_is_c99():
    _build()
    out = subprocess.run([os.path.join(BUILD, "c99_header")], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "c99 header ok" in out.stdout


def test_cpp_dropin_without_device():
    if not _ref_available():
        pytest.skip("the C++ drop-in test compiles against the reference's headers, absent here")
    _build()
    out = subprocess.run([os.path.join(BUILD, "dropin_test"), "nodevice"], capture_output=True, text=True,
                         timeout=120, env={**os.environ, "CUDA_VISIBLE_DEVICES": ""})
    assert out.returncode == 0, out.stdout + out.stderr


@pytest.mark.parametrize("case,message", [(1, "device preconditioners"), (2, "runs only inside")])
def test_cpp_dropin_misuse_does_not_compile(case, message):
    if not _ref_available():
        pytest.skip("the C++ drop-in test compiles against the reference's headers, absent here")
    import sysconfig
    json_inc = os.path.join(sysconfig.get_paths()["purelib"], "include", "cudnn_frontend", "thirdparty")
    cmd = ["g++", "-std=c++20", "-fsyntax-only", f"-DMISUSE={case}", "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(ROOT, "oracle", "_ref", "gen"), "-I", REF, "-I", json_inc,
           os.path.join(CPP, "misuse.cpp")]
    ok = subprocess.run(cmd[:3] + ["-DMISUSE=0"] + cmd[4:], capture_output=True, text=True, timeout=300)
    assert ok.returncode == 0, ok.stderr[-2000:]
    bad = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert bad.returncode != 0 and message in bad.stderr, bad.stderr[-2000:]


@pytest.mark.gpu
def test_cpp_dropin_on_gpu():
    exe = os.path.join(BUILD, "dropin_test")
    assert os.path.isfile(exe), "tests/cpp/_build/dropin_test is built by tests/cpp/build.sh where the reference is"
    out = subprocess.run([exe, "gpu"], capture_output=True, text=True, timeout=600)
    print(out.stdout)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "all checks passed" in out.stdout
