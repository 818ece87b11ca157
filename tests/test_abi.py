"""The C ABI: the library loads on a machine without a GPU and exports every entry point of include/*.h."""

import ctypes
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def declared() -> list[str]:
    names = []
    for h in sorted((ROOT / "include").glob("*.h")):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*(cb_[a-z_0-9]+)\s*\(", text, flags=re.M)
    return names


def test_library_exports_every_declared_symbol():
    from cubam_b200 import _lib

    names = declared()
    assert len(names) >= 20
    lib = ctypes.CDLL(str(_lib.LIB_PATH))
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) <= set(_lib.exported_symbols()) | set(), set(names) - set(_lib.exported_symbols())


def test_no_gpu_calls_needed_for_sizes():
    from cubam_b200 import _lib

    assert _lib.lib.cb_version().startswith(b"cubam_b200")
    assert _lib.lib.cb_scan_workspace_bytes(1 << 20) > (1 << 20) // 28 * 8
    assert _lib.lib.cb_record_chain_workspace_bytes(1 << 20) > 0
    assert _lib.lib.cb_inflate_workspace_bytes() >= 8
    assert ctypes.sizeof(_lib.MemberJob) == 32
    assert ctypes.sizeof(_lib.ScanSummary) == 48
    assert ctypes.sizeof(_lib.InflateSummary) == 24
    assert ctypes.sizeof(_lib.ChainSummary) == 32


def test_bad_arguments_are_rejected_without_a_launch():
    from cubam_b200 import _lib

    assert _lib.lib.cb_scan_members(None, -1, 0, 0, None, 0, None, None, 0, None) == _lib.ARG
    assert _lib.lib.cb_inflate(None, -1, None, None, 1, None, None, None, 0, None) == _lib.ARG
    assert _lib.lib.cb_find_tags(None, None, 1, b"CB", 0, None, None, None, None, None) == _lib.ARG
    assert _lib.lib.cb_decode_fixed(None, None, -5, *([None] * 11), None) == _lib.ARG


def test_launch_parameters_are_checked_and_restored():
    from cubam_b200 import _lib

    L = _lib.lib
    assert L.cb_get_param(_lib.PARAM_CHAIN_TILE) == 0
    assert L.cb_get_param(99) == -1
    assert L.cb_set_param(99, 1) == _lib.ARG
    assert L.cb_set_param(_lib.PARAM_CHAIN_TILE, 3000) == _lib.ARG  # not a power of two
    assert L.cb_set_param(_lib.PARAM_CHAIN_TILE, 1 << 17) == _lib.ARG  # above 64 KiB
    assert L.cb_set_param(_lib.PARAM_COPY_WARPS, 4) == _lib.ARG
    assert L.cb_set_param(_lib.PARAM_COPY_UNITS, 3) == _lib.ARG
    assert L.cb_set_param(_lib.PARAM_CHAIN_TILE, 8192) == _lib.OK
    assert L.cb_get_param(_lib.PARAM_CHAIN_TILE) == 8192
    assert L.cb_set_param(_lib.PARAM_CHAIN_TILE, 1024) == _lib.ARG
    assert L.cb_set_param(_lib.PARAM_CHAIN_TILE, -1) == _lib.OK
    assert L.cb_get_param(_lib.PARAM_CHAIN_TILE) == 0
    for key, default in ((_lib.PARAM_INFLATE_FORM, 3), (_lib.PARAM_DECODE_ROOT, 7), (_lib.PARAM_COPY_WARPS, 12),
                         (_lib.PARAM_DECODE_STEPS, 16), (_lib.PARAM_DECODE_PREFETCH, 4),
                         (_lib.PARAM_SPLIT_MIN_JOBS, 8192), (_lib.PARAM_COPY_UNITS, 2),
                         (_lib.PARAM_DECODE_PIPELINE, 1)):
        assert L.cb_get_param(key) == default


def test_header_compiles_as_c_and_a_c_program_links(tmp_path):
    """include/cubam_b200.h is plain C99, and a C program links the library and calls it (entry points
    that need no GPU: the version, the launch parameters, the workspace sizes)."""
    import shutil
    import subprocess

    from cubam_b200 import _lib

    gcc = shutil.which("gcc")
    if gcc is None:
        import pytest

        pytest.skip("no C compiler")
    src = tmp_path / "use.c"
    src.write_text(r'''
#include <stdio.h>
#include "cubam_b200.h"
int main(void) {
    cb_batch* none = 0;
    (void)none;
    if (cb_get_param(CB_PARAM_INFLATE_FORM) != 3) return 2;
    if (cb_set_param(CB_PARAM_DECODE_ROOT, 6) != CB_OK || cb_get_param(CB_PARAM_DECODE_ROOT) != 6) return 3;
    if (cb_set_param(CB_PARAM_DECODE_ROOT, 9) != CB_ERR_ARG) return 4;
    if (cb_scan_workspace_bytes(1 << 20) == 0 || cb_record_chain_workspace_bytes(1 << 20) == 0) return 5;
    if (cb_inflate_split_workspace_bytes(10, 655360) < 2 * 655360) return 6;
    printf("%s\n", cb_version());
    return 0;
}
''')
    exe = tmp_path / "use"
    libdir = Path(_lib.LIB_PATH).parent
    subprocess.run([gcc, "-std=c99", "-Wall", "-Werror", "-I", str(ROOT / "include"), str(src), "-o", str(exe),
                    "-L", str(libdir), "-lcubam_b200", f"-Wl,-rpath,{libdir}"], check=True, capture_output=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, (r.returncode, r.stderr)
    assert r.stdout.strip()
