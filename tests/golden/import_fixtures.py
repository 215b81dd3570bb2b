"""Copy vaco's checked-in dav1d golden vectors for the AV1 post-filters into
tests/golden/ (gzip-compressed) and record their SHA-256 in MANIFEST.txt.

The vectors are output data produced by vaco's own oracle scripts from the
pinned BSD-2-Clause dav1d revision aa09a630ef57ee7d9482ffb7ef355a903dbb5302
(vaco: scripts/gen-av1-cdef-oracle.py:13, provenance/vaco-codec-av1-*.toml).
They are the only pins for the restated CDEF, superres and restoration
arithmetic.  Run once in a checkout next to the vaco sources:

    python tests/golden/import_fixtures.py /path/to/vaco
"""
import gzip
import hashlib
import pathlib
import sys

FIXTURES = {
    # vaco path (relative)                                                       -> local name
    "crates/tool/vaco-checkasm/tests/fixtures/av1-cdef-dav1d.bin": "av1-cdef-dav1d.bin.gz",
    "crates/codec/vaco-codec-av1/tests/fixtures/superres-dav1d.u16le": "superres-dav1d.u16le.gz",
    "crates/codec/vaco-codec-av1/tests/fixtures/restoration-dav1d-8.u16le": "restoration-dav1d-8.u16le.gz",
    "crates/codec/vaco-codec-av1/tests/fixtures/restoration-dav1d-high.u16le": "restoration-dav1d-high.u16le.gz",
    "crates/codec/vaco-codec-av1/tests/fixtures/restoration-constant-8.u16le": "restoration-constant-8.u16le.gz",
    "crates/codec/vaco-codec-av1/tests/fixtures/restoration-constant-high.u16le": "restoration-constant-high.u16le.gz",
}


def main() -> None:
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/import_fixtures.py /path/to/vaco")
    root = pathlib.Path(sys.argv[1])
    here = pathlib.Path(__file__).resolve().parent
    lines = []
    for rel, name in FIXTURES.items():
        raw = (root / rel).read_bytes()
        (here / name).write_bytes(gzip.compress(raw, compresslevel=9, mtime=0))
        lines.append(f"{hashlib.sha256(raw).hexdigest()}  {len(raw)}  {name}  {rel}")
    (here / "MANIFEST.txt").write_text("\n".join(lines) + "\n")


if __name__ == "__main__":
    main()
