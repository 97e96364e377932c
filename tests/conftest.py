"""Shared test setup: the `gpu` marker, in-tree builds and the TAL-SH session on GPU 0."""
import ctypes as C
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an NVIDIA B200 (sm_100a) GPU")


@pytest.fixture(scope="session")
def built():
    """Builds libtalsh.so and liboracle.so in-tree when their sources are newer."""
    from tal_sh_b200.build import build_library
    from oracle.build import build_oracle
    build_library()
    build_oracle()
    return True


@pytest.fixture(scope="session")
def talsh(built):
    """TAL-SH initialized on GPU 0 for the whole GPU session (fails loudly without a GPU)."""
    import tal_sh_b200 as T
    L = T.lib()
    n = C.c_int(0)
    assert L.talshDeviceCount(T.DEV_NVIDIA_GPU, C.byref(n)) == 0
    if n.value < 1:
        pytest.fail("GPU tests need a CUDA device; none is visible")
    hbuf = C.c_size_t(1 << 24)
    harg = C.c_int(0)
    rc = L.talshInit(C.byref(hbuf), C.byref(harg), 1, T.ivec([0]), 0, None, 0, None)
    assert rc == 0, rc
    yield L
    assert L.talshShutdown() == 0
