"""The JNI glue (gravity_b200/jni/gravity_p3m_jni.c) compiles and forwards to
the C-ABI. No JDK is installed here, so it is compiled against a minimal
<jni.h> stand-in (tests/jni_stub/jni.h) and driven through a fake JNI
environment (tests/jni_stub/harness.c) that calls the glue's
Java_dev_gravity_P3mNative_* functions as the JVM would. Without a GPU the
calls take the library's argument and no-device error paths; nothing
launches a kernel.
"""

import ctypes
import shutil
import subprocess
from pathlib import Path

import pytest

from gravity_b200 import _abi

REPO = Path(__file__).resolve().parent.parent
STUB = REPO / "tests" / "jni_stub"
GLUE = REPO / "gravity_b200" / "jni" / "gravity_p3m_jni.c"


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.fail("a C compiler is required to build the JNI glue")
    lib = _abi.load()  # builds libgravity_p3m.so when needed
    out = tmp_path_factory.mktemp("jni") / "libharness.so"
    cmd = [cc, "-O2", "-Wall", "-Wextra", "-Werror", "-shared", "-fPIC", "-I", str(STUB),
           "-I", str(REPO / "include"), str(GLUE), str(STUB / "harness.c"),
           "-L", str(_abi.library_path().parent), "-lgravity_p3m",
           f"-Wl,-rpath,{_abi.library_path().parent}", "-o", str(out)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    h = ctypes.CDLL(str(out))
    h.harness_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_longlong),
                                 ctypes.c_char_p, ctypes.c_int]
    h.harness_destroy.argtypes = [ctypes.c_longlong]
    h.harness_download.argtypes = [ctypes.c_longlong, ctypes.c_int, ctypes.c_void_p]
    h.harness_step.argtypes = [ctypes.c_longlong, ctypes.c_int, ctypes.c_int]
    h.harness_step_io.argtypes = [ctypes.c_longlong, ctypes.c_int, ctypes.c_void_p,
                                  ctypes.c_void_p]
    del lib
    return h


def _create(h, w, hgt):
    handle = ctypes.c_longlong(-1)
    msg = ctypes.create_string_buffer(256)
    st = h.harness_create(w, hgt, ctypes.byref(handle), msg, 256)
    return st, handle.value, msg.value.decode()


def test_create_rejects_an_invalid_grid_through_the_glue(harness):
    st, handle, msg = _create(harness, 500, 256)
    assert st == _abi.P3M_ERR_UNSUPPORTED
    assert handle == 0
    assert "grid" in msg


def test_create_and_destroy_through_the_glue(harness):
    st, handle, msg = _create(harness, 512, 256)
    if st == _abi.P3M_OK:  # a GPU is present
        assert handle != 0
        assert harness.harness_destroy(handle) == _abi.P3M_OK
    else:  # no device: the library's CUDA error, surfaced with its message
        assert st == _abi.P3M_ERR_CUDA, (st, msg)
        assert handle == 0 and msg


def test_null_context_calls_are_argument_errors(harness):
    assert harness.harness_destroy(0) == _abi.P3M_OK
    buf = (ctypes.c_float * 16)()
    assert harness.harness_download(0, 4, ctypes.cast(buf, ctypes.c_void_p)) == _abi.P3M_ERR_INVALID_ARGUMENT
    assert harness.harness_step(0, 4, 1) == _abi.P3M_ERR_INVALID_ARGUMENT
    assert harness.harness_step_io(0, 4, ctypes.cast(buf, ctypes.c_void_p),
                                   ctypes.cast(buf, ctypes.c_void_p)) == _abi.P3M_ERR_INVALID_ARGUMENT
