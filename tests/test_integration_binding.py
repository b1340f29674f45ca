"""The Rust FFI declarations a maintainer copies from INTEGRATION.md match
include/gpv.h: every `#[repr(C)]` record there has the header's field names,
types and order, and the layout those Rust types imply (sizes, alignments,
offsets) is what a C compiler gives the header's structs -- checked by
compiling a program that includes gpv.h and `static_assert`s every size and
offset.  A record that drifts in either file fails here."""
import os
import re
import shutil
import subprocess

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "gpv.h")
DOC = os.path.join(ROOT, "INTEGRATION.md")

# Rust type -> (size, align, canonical kind) for the types the binding uses
RUST_SCALARS = {"f64": (8, 8, "f64"), "f32": (4, 4, "f32"), "i32": (4, 4, "i32"), "u32": (4, 4, "u32"),
                "i64": (8, 8, "i64"), "u64": (8, 8, "u64"), "usize": (8, 8, "u64"), "u8": (1, 1, "u8")}
C_SCALARS = {"double": "f64", "float": "f32", "int32_t": "i32", "uint32_t": "u32", "int64_t": "i64",
             "uint64_t": "u64", "size_t": "u64", "uint8_t": "u8"}


def rust_records():
    """name -> [(field, kind, count)] for every #[repr(C)] struct with fields."""
    text = open(DOC).read()
    out = {}
    for m in re.finditer(r"#\[repr\(C\)\](?:\s*#\[derive\([^)]*\)\])*\s*pub struct (\w+)\s*\{(.*?)\}", text, re.S):
        name, body = m.group(1), m.group(2)
        fields = []
        for fm in re.finditer(r"pub (\w+):\s*([^,]+?)\s*(?:,|$)", body.strip() + ","):
            fname, ty = fm.group(1), fm.group(2).strip()
            arr = re.fullmatch(r"\[(\w+);\s*(\d+)\]", ty)
            if arr:
                fields.append((fname, RUST_SCALARS[arr.group(1)][2], int(arr.group(2))))
            elif ty.startswith("*") or ty.startswith("Option<") or ty.endswith("_fn"):
                fields.append((fname, "ptr", 1))
            else:
                fields.append((fname, RUST_SCALARS[ty][2], 1))
        if fields:
            out[name] = fields
    return out


def c_records():
    """name -> [(field, kind, count)] for every `typedef struct { ... } name;`."""
    text = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    out = {}
    for m in re.finditer(r"typedef struct\s*\{(.*?)\}\s*(\w+)\s*;", text, re.S):
        body, name = m.group(1), m.group(2)
        fields = []
        for decl in body.split(";"):
            decl = decl.strip()
            if not decl:
                continue
            dm = re.fullmatch(r"(?:const\s+)?([\w]+)\s*(\**)\s*(.*)", decl, re.S)
            base, star, names = dm.group(1), dm.group(2), dm.group(3)
            for nm in names.split(","):
                nm = nm.strip()
                ptr = star or nm.startswith("*") or base.endswith("_fn")
                nm = nm.lstrip("*").strip()
                am = re.fullmatch(r"(\w+)\[(\d+)\]", nm)
                count = int(am.group(2)) if am else 1
                nm = am.group(1) if am else nm
                # a nested record keeps its type name (no binding declares one)
                fields.append((nm, "ptr" if ptr else C_SCALARS.get(base, base), count))
        out[name] = fields
    return out


def layout(fields):
    """C layout of a record: field offsets, size, align (repr(C) rules)."""
    sizes = {"f64": 8, "f32": 4, "i32": 4, "u32": 4, "i64": 8, "u64": 8, "u8": 1, "ptr": 8}
    off, align, offs = 0, 1, {}
    for name, kind, count in fields:
        s = sizes[kind]
        off = (off + s - 1) // s * s
        offs[name] = off
        off += s * count
        align = max(align, s)
    return offs, (off + align - 1) // align * align


def test_rust_records_match_the_header():
    rust, c = rust_records(), c_records()
    assert {"gpv_subset_desc", "gpv_solve_params", "gpv_subset_result", "gpv_mesh_params",
            "gpv_mesh_stats"} <= set(rust)
    for name, fields in rust.items():
        assert name in c, f"{name} is not a record of gpv.h"
        assert fields == c[name], f"{name}: INTEGRATION.md {fields} != gpv.h {c[name]}"


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs a C compiler")
def test_header_layout_is_the_rust_layout(tmp_path):
    """Compiles `static_assert(sizeof / offsetof == the Rust-implied value)`
    for every record the binding declares, then runs the program."""
    rust = rust_records()
    lines = ["#include <stddef.h>", "#include <stdio.h>", "#include <assert.h>", '#include "gpv.h"', "int main(void) {"]
    for name, fields in rust.items():
        offs, size = layout(fields)
        lines.append(f'    static_assert(sizeof({name}) == {size}, "{name} size");')
        for f, _, _ in fields:
            lines.append(f'    static_assert(offsetof({name}, {f}) == {offs[f]}, "{name}.{f} offset");')
        lines.append(f'    printf("{name} %zu\\n", sizeof({name}));')
    lines += ["    return 0;", "}"]
    src = tmp_path / "abi_layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "abi_layout"
    r = subprocess.run(["gcc", "-std=c11", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src),
                        "-o", str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    sizes = dict(zip(out[::2], map(int, out[1::2])))
    assert sizes["gpv_subset_desc"] == 120 and sizes["gpv_subset_result"] == 200
    assert sizes["gpv_solve_params"] == 48 and sizes["gpv_mesh_params"] == 208


def test_ctypes_mirror_matches_the_header(gpv_mod):
    """The Python binding's record mirrors have the header's sizes too."""
    import ctypes as ct

    from gpv import _lib
    c = c_records()
    assert layout(c["gpv_subset_desc"])[1] == _lib.DESC_DTYPE.itemsize
    assert layout(c["gpv_subset_result"])[1] == _lib.RESULT_DTYPE.itemsize
    assert [f for f, _, _ in c["gpv_subset_result"]] == list(_lib.RESULT_DTYPE.names)
    for rec, mirror in (("gpv_solve_params", _lib.SolveParams), ("gpv_mesh_params", _lib.MeshParams),
                        ("gpv_mesh_stats", _lib.MeshStats), ("gpv_peaks", _lib.Peaks)):
        offs, size = layout(c[rec])
        assert ct.sizeof(mirror) == size, rec
        assert [f for f, _ in mirror._fields_] == [f for f, _, _ in c[rec]], rec
        for f, _ in mirror._fields_:
            assert getattr(mirror, f).offset == offs[f], (rec, f)
