"""The Rust FFI crate (crates/hw/vaco-hw-cuda-av1) against the C header it
binds: this image has no Rust toolchain, so these checks stand in for the
compiler on the parts that must match -- every entry point of
include/vaco_av1_gpu.h is declared with the same number of parameters, every
#[repr(C)] struct lists the header's fields in the header's order, and the
message table is the library's."""
import pathlib
import re

import pytest

from vaco_b200 import abi

ROOT = pathlib.Path(__file__).resolve().parent.parent
CRATE = ROOT / "crates" / "hw" / "vaco-hw-cuda-av1"
HEADER = (ROOT / "include" / "vaco_av1_gpu.h").read_text()
FFI = (CRATE / "src" / "ffi.rs").read_text()


def header_prototypes():
    text = re.sub(r"/\*.*?\*/", "", HEADER, flags=re.S)
    out = {}
    for ret, args in re.findall(r"VACO_AV1_API\s+([^;]+?)\s*\(([^;]*?)\)\s*;", text, flags=re.S):
        name = re.search(r"(vaco_av1_\w+)$", " ".join(ret.split())).group(1)
        out[name] = len([a for a in args.split(",") if a.strip()])
    return out


def rust_prototypes():
    return {m.group(1): len([a for a in m.group(2).split(",") if a.strip()])
            for m in re.finditer(r"pub fn (vaco_av1_\w+)\(([^)]*)\)", FFI)}


def test_every_entry_point_is_declared_with_its_arity():
    c, rust = header_prototypes(), rust_prototypes()
    assert len(c) >= 45
    assert set(c) == set(rust)
    for name, n in c.items():
        assert rust[name] == n, name


def header_struct_fields(cname):
    body = re.search(r"typedef struct " + cname + r" \{(.*?)\} " + cname + ";", HEADER, flags=re.S).group(1)
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    names = []
    for decl in body.split(";"):
        decl = decl.strip()
        if not decl:
            continue
        for part in decl.split(","):
            m = re.search(r"(\w+)\s*(\[\w+\])?\s*$", part.strip())
            names.append(m.group(1))
    return names


def rust_struct_fields(rname):
    body = re.search(r"pub struct " + rname + r" \{(.*?)\n\}", FFI, flags=re.S).group(1)
    return [m.group(1) for m in re.finditer(r"pub (\w+):", body)]


@pytest.mark.parametrize("cname,rname", [
    ("vaco_av1_picture", "Picture"), ("vaco_av1_frame_info", "FrameInfo"), ("vaco_av1_cdef_params", "CdefParams"),
    ("vaco_av1_cdef_filter_params", "CdefFilterParams"),
    ("vaco_av1_superres_picture_config", "SuperresPictureConfig"), ("vaco_av1_lr_unit", "LrUnit"),
    ("vaco_av1_lr_plane_config", "LrPlaneConfig"), ("vaco_av1_deblock_params", "DeblockParams"),
    ("vaco_av1_frame_job", "FrameJob"), ("vaco_av1_tuning", "Tuning"), ("vaco_av1_server_config", "ServerConfig"),
    ("vaco_av1_server_stats", "ServerStats"), ("vaco_av1_frame_buffer", "FrameBuffer"),
    ("vaco_av1_film_grain_params", "FilmGrainParams"),
])
def test_repr_c_structs_follow_the_header(cname, rname):
    c = header_struct_fields(cname)
    rust = ["type" if f == "kind" else f for f in rust_struct_fields(rname)]  # `type` is a Rust keyword
    assert rust == c


def test_message_table_is_the_librarys():
    table = re.search(r"pub const MESSAGES: \[&str; (\d+)\] = \[(.*?)\];", FFI, flags=re.S)
    texts = re.findall(r'"((?:[^"\\]|\\.)*)"', table.group(2))
    assert int(table.group(1)) == len(texts) == len(abi.MESSAGES)
    assert texts == [abi.MESSAGES[i] for i in range(len(texts))]


def test_crate_sits_in_the_unsafe_allowed_family_with_its_lints():
    manifest = (CRATE / "Cargo.toml").read_text()
    assert 'name = "vaco-hw-cuda-av1"' in manifest  # xtask unsafe_audit allows the vaco-hw- prefix
    assert 'undocumented_unsafe_blocks = "deny"' in manifest
    lib = (CRATE / "src" / "lib.rs").read_text()
    # every unsafe block or impl is preceded by a SAFETY comment
    lines = lib.splitlines()
    for i, ln in enumerate(lines):
        if re.search(r"\bunsafe\s*(\{|impl)", ln) and "SAFETY" not in ln:
            window = "\n".join(lines[max(0, i - 6):i])
            assert "SAFETY:" in window, f"lib.rs:{i + 1}"
