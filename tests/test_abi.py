"""The C-ABI library loads without a GPU and exports every declared symbol."""

import ctypes
import re

from conftest import ROOT


def _declared_symbols():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(ssm_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_header_declares_entry_points():
    names = _declared_symbols()
    assert {"ssm_ddm_flexbound", "ssm_ddm", "ssm_levy_flexbound", "ssm_version"} <= names


def test_library_exports_every_declared_symbol():
    from ssms_b200 import _lib

    lib = _lib.lib()
    raw = ctypes.CDLL(str(_lib._LIB_PATH))
    missing = [n for n in sorted(_declared_symbols()) if not hasattr(raw, n)]
    assert not missing, f"symbols declared in include/ but not exported: {missing}"
    assert set(_lib.exported_symbols()) <= _declared_symbols()
    assert lib.ssm_version() >= 100


def test_workspace_query_needs_no_device():
    from ssms_b200 import _lib

    lib = _lib.lib()
    assert lib.ssm_ddm_workspace_bytes(0) >= 256
    assert lib.ssm_ddm_workspace_bytes(4096) >= 256 + 4096 * 64
    assert lib.ssm_ddm_workspace_bytes(4096) % 256 == 0


def test_argument_errors_are_reported_without_a_launch():
    """Invalid arguments are rejected before any CUDA call (ValueError in Python)."""
    import pytest

    from ssms_b200 import _lib

    lib = _lib.lib()
    st = lib.ssm_ddm_flexbound(None, None, None, None, None, None, 1, 1, None, 20.0, None, 0.001,
                               _lib.BOUND_CONSTANT, None, None, None, 0, 0, 0, 0, None, 0, None,
                               None, None, None, None, 0, None, None, 0, None)
    assert st == _lib.SSM_ERR_ARG
    assert b"required" in lib.ssm_last_error()
    with pytest.raises(ValueError):
        _lib.check(st)


def test_launch_struct_layout_matches_the_header(tmp_path):
    """ctypes' SsmLaunch has the size and field offsets the C compiler gives ssm_launch."""
    import shutil
    import subprocess

    import pytest

    from ssms_b200 import _lib

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    fields = [f for f, _ in _lib.SsmLaunch._fields_]
    src = tmp_path / "layout.c"
    src.write_text("#include <stddef.h>\n#include <stdio.h>\n#include \"ssm_b200.h\"\nint main(void) {\n"
                   "  printf(\"%zu\\n\", sizeof(ssm_launch));\n"
                   + "".join(f"  printf(\"%zu\\n\", offsetof(ssm_launch, {f}));\n" for f in fields)
                   + "  return 0;\n}\n")
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    assert got[0] == ctypes.sizeof(_lib.SsmLaunch)
    assert got[1:] == [getattr(_lib.SsmLaunch, f).offset for f in fields]
    assert getattr(_lib.SsmLaunch, "first_trial").offset == 16  # unchanged by refill_min (padding slot)
    # lanes_per_walk was appended: every earlier field keeps its offset
    assert getattr(_lib.SsmLaunch, "lanes_per_walk").offset == 40
    assert ctypes.sizeof(_lib.SsmLaunch) == 48
