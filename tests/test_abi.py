"""The C-ABI library loads and exports every entry point include/*.h declares,
and the ctypes structs match the header's layout (no GPU needed)."""
import ctypes
import pathlib
import re

import oracle
from vaco_b200 import abi, _lib

ROOT = pathlib.Path(__file__).resolve().parent.parent


def declared_functions():
    names = []
    for h in (ROOT / "include").glob("*.h"):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(vaco_av1_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    lib = _lib.lib()  # raises if the library was not built
    declared = declared_functions()
    assert len(declared) >= 19
    for name in declared:
        assert hasattr(lib, name), name
    assert set(declared) == set(_lib.exported_symbols())


def test_message_table_matches_library():
    lib = _lib.lib()
    for mid, text in abi.MESSAGES.items():
        assert lib.vaco_av1_message(mid).decode() == text


def test_ctypes_struct_layout_matches_gcc():
    l = oracle.lib()
    l.vo_sizeof.argtypes = [ctypes.c_char_p]
    for name, size in abi.STRUCT_SIZES.items():
        assert l.vo_sizeof(name.encode()) == size, name


def test_context_without_gpu_reports_device_error():
    import torch
    if torch.cuda.is_available():
        return
    h = ctypes.c_void_p()
    assert _lib.lib().vaco_av1_ctx_create(0, ctypes.byref(h)) == abi.DEVICE_ERROR
