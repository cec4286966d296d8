"""The C-ABI library loads on a machine without a GPU and exports every
symbol include/gcr.h declares (no compute calls here)."""
import ctypes
import os
import re

from gliding_collective_rotation_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    with open(os.path.join(ROOT, "include", "gcr.h")) as fh:
        hdr = fh.read()
    return re.findall(r"^GCR_API (?:int|const char \*) ?\*?(gcr_\w+)\(", hdr, re.M)


def test_header_symbols_exported():
    lib = ctypes.CDLL(_lib.LIB_PATH)
    names = _declared()
    assert len(names) >= 17
    for n in names:
        assert hasattr(lib, n), n


def test_binding_covers_header():
    assert set(_declared()) == set(_lib.SIGNATURES)


def test_version_and_error_string_without_gpu():
    lib = _lib.load()
    assert lib.gcr_version() >= 1
    # a call that fails argument checks before touching the device
    rc = lib.gcr_philox_noise(5, 0, 0, 1, 1, 1, None, None)
    assert rc == -1
    assert b"bad argument" in lib.gcr_last_error()


def test_structs_match_header_sizes(tmp_path):
    """The ctypes mirrors have the sizes and field offsets the C compiler
    gives the header structs."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        import pytest
        pytest.skip("no C compiler")
    src = tmp_path / "sizes.c"
    src.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "gcr.h"\n'
        'int main(){printf("%zu %zu %zu %zu %zu %zu %zu\\n", sizeof(gcr_config), sizeof(gcr_system_desc),'
        ' sizeof(gcr_system_buffers), sizeof(gcr_call), sizeof(gcr_status),'
        ' offsetof(gcr_system_desc, seed), offsetof(gcr_config, ctas_per_sm)); return 0;}\n')
    exe = tmp_path / "sizes"
    subprocess.run([cc, "-I", os.path.join(ROOT, "include"), "-o", str(exe), str(src)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    want = [ctypes.sizeof(_lib.Config), ctypes.sizeof(_lib.SystemDesc), ctypes.sizeof(_lib.SystemBuffers),
            ctypes.sizeof(_lib.Call), ctypes.sizeof(_lib.Status), _lib.SystemDesc.seed.offset,
            _lib.Config.ctas_per_sm.offset]
    assert got == want
