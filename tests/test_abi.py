"""CPU tests of the C-ABI library: it loads, exports every declared symbol,
validates arguments without a device, and its host-side generators agree
with the oracle's."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lib(hw):
    if not os.path.exists(hw.LIB_PATH):
        from hila_b200 import build
        build.build()
    return hw.load_library()


def declared_symbols():
    names = set()
    inc = os.path.join(ROOT, "include")
    for fn in os.listdir(inc):
        if not fn.endswith(".h"):
            continue
        src = open(os.path.join(inc, fn)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names |= set(re.findall(r"\b(hw_[a-z0-9_]+)\s*\(", src))
    return sorted(names)


def test_every_declared_symbol_is_exported(lib):
    names = declared_symbols()
    assert len(names) >= 25
    for n in names:
        assert hasattr(lib, n), f"{n} declared in include/ but not exported"


def test_python_binding_covers_header(hw, lib):
    missing = set(declared_symbols()) - set(hw.exported_symbols())
    assert not missing, f"python binding lacks {sorted(missing)}"


def test_api_version(hw, lib):
    assert lib.hw_api_version() == hw.API_VERSION == 2


def test_no_device_fails_loudly(hw, lib):
    if hw.device_count() > 0:
        pytest.skip("a CUDA device is present")
    with pytest.raises(hw.HilaError) as e:
        hw.Context(0)
    assert e.value.code == hw.HW_ERR_NO_DEVICE


def test_generate_rejects_bad_dims(hw, lib):
    with pytest.raises(hw.HilaError):
        hw.generate_links((3, 4, 4, 4), 0.3, 1)


def test_generators_match_oracle(hw, oracle):
    dims = (4, 4, 2, 6)
    U1 = hw.generate_links(dims, 0.3, 17)
    U2 = oracle.gen_links(dims, 0.3, 17)
    assert np.abs(U1 - U2).max() < 1e-14
    for par in (oracle.EVEN, oracle.ODD, oracle.ALL):
        s1 = hw.generate_spinor(dims, 5, par)
        s2 = oracle.gen_spinor(dims, 5, par)
        assert np.array_equal(s1, s2)


C_CONSUMER = r"""
#include "hila_b200.h"
#include <stdio.h>
#include <stdlib.h>
int main(void) {
    int dims[4] = {4, 4, 4, 2};
    double *U = malloc(sizeof(double) * 4 * 128 * 18);
    int rc = hw_generate_links(dims, 0.3, 7, U);
    printf("%d %d %.17g %.17g\n", hw_api_version(), rc, U[0], U[4 * 128 * 18 - 1]);
    free(U);
    return rc;
}
"""


def test_header_is_c99_and_links_from_c(hw, lib, tmp_path):
    """A plain C program (no C++) includes the header under -std=c99 -pedantic, links the
    library and calls it: what a cgo or C caller sees."""
    import shutil
    import subprocess
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("gcc not available")
    src = tmp_path / "consumer.c"
    src.write_text(C_CONSUMER)
    exe = tmp_path / "consumer"
    libdir = os.path.dirname(hw.LIB_PATH)
    libname = os.path.basename(hw.LIB_PATH)[3:-3]
    cc = subprocess.run([gcc, "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", "-I",
                         os.path.join(ROOT, "include"), str(src), "-L", libdir, "-l" + libname,
                         "-Wl,-rpath," + libdir, "-o", str(exe)], capture_output=True, text=True)
    assert cc.returncode == 0, cc.stderr
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert run.returncode == 0, run.stderr
    version, rc, first, last = run.stdout.split()
    assert int(rc) == 0 and int(version) == hw.API_VERSION
    U = hw.generate_links((4, 4, 4, 2), 0.3, 7)
    assert float(first) == U.reshape(-1)[0] and float(last) == U.reshape(-1)[-1]
