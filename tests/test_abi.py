"""The C-ABI library loads and exports every symbol include/*.h declares (CPU only)."""
from __future__ import annotations

import ctypes
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols() -> set[str]:
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        txt = h.read_text()
        names |= set(re.findall(r"^FF_API\s+[\w\s\*]+?\b(ff_\w+)\s*\(", txt, flags=re.M))
    return names


def test_header_declares_entry_points():
    names = declared_symbols()
    for must in ["ff_context_create", "ff_scene_create", "ff_trace", "ff_render", "ff_film_read"]:
        assert must in names


def test_library_exports_every_declared_symbol(ff_lib):
    from firefly_b200 import _abi
    names = declared_symbols()
    missing = [n for n in sorted(names) if not hasattr(ff_lib, n)]
    assert not missing, f"not exported: {missing}"
    # the ctypes table covers the same set
    assert names == set(_abi.SIGNATURES), names ^ set(_abi.SIGNATURES)


def test_context_create_without_device_reports_status(ff_lib):
    from tests.conftest import has_gpu
    if has_gpu():
        return
    h = ctypes.c_void_p()
    st = ff_lib.ff_context_create(None, ctypes.byref(h))
    assert st != 0 and not h.value
    assert isinstance(ff_lib.ff_last_error_message(None), bytes)


def test_null_arguments_are_rejected(ff_lib):
    assert ff_lib.ff_context_create(None, None) == 1
    assert ff_lib.ff_context_destroy(None) == 1
    assert ff_lib.ff_scene_destroy(None) == 1
    assert ff_lib.ff_film_destroy(None) == 1
    assert ff_lib.ff_trace(None, None, None, 0, None, 0) == 1


def test_struct_layouts_match_the_header(tmp_path):
    """Every struct the ctypes table mirrors has the header's size and field
    offsets (a C program compiled from include/firefly_b200.h prints them)."""
    import shutil
    import subprocess

    import pytest

    from firefly_b200 import _abi
    if not shutil.which("gcc"):
        pytest.skip("gcc not available")
    structs = {n: getattr(_abi, n) for n in dir(_abi)
               if n.startswith("ff_") and isinstance(getattr(_abi, n), type)
               and issubclass(getattr(_abi, n), ctypes.Structure)}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "firefly_b200.h"', "int main(void) {"]
    for n, cls in sorted(structs.items()):
        lines.append(f'printf("{n} size %zu\\n", sizeof({n}));')
        for f, *_ in cls._fields_:
            lines.append(f'printf("{n} {f} %zu\\n", offsetof({n}, {f}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    got = {}
    for ln in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines():
        a, b, c = ln.split()
        got[(a, b)] = int(c)
    bad = []
    for n, cls in structs.items():
        if got[(n, "size")] != ctypes.sizeof(cls):
            bad.append(f"{n}: size {got[(n, 'size')]} vs ctypes {ctypes.sizeof(cls)}")
        for f, *_ in cls._fields_:
            if got[(n, f)] != getattr(cls, f).offset:
                bad.append(f"{n}.{f}: offset {got[(n, f)]} vs ctypes {getattr(cls, f).offset}")
    assert not bad, bad


def test_debug_hooks_need_no_device(ff_lib):
    """The allocation counters and the refusal switch work without a GPU."""
    total, live = ctypes.c_uint64(7), ctypes.c_int64(7)
    assert ff_lib.ff_debug_alloc_stats(ctypes.byref(total), ctypes.byref(live)) == 0
    assert total.value >= 0
    assert ff_lib.ff_debug_alloc_stats(None, None) == 0
    assert ff_lib.ff_debug_fail_alloc_after(3) == 0
    assert ff_lib.ff_debug_fail_alloc_after(-1) == 0
    assert ff_lib.ff_debug_cache_wait_limit(None, 0) == 1
