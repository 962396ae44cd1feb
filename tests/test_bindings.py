"""The Rust declarations (lbm-arrayfire_b200/bindings/lbm_sys.rs) and a plain-C caller
(bindings/c_abi_check.c) against include/lbm.h.

Rust cannot be compiled here, so the Rust file is checked by reading it: every function of the
header is declared with the same parameter and return types, the #[repr(C)] structs list the header's
fields in order with matching types, and the sizes and offsets the Rust file asserts are the ones gcc
gives the header (the C program prints them).  On a GPU the C program also steps a lattice."""
import re
import subprocess

import numpy as np
import pytest

from helpers import O, P, ROOT

HEADER = ROOT / "include" / "lbm.h"
RUST = ROOT / "lbm-arrayfire_b200" / "bindings" / "lbm_sys.rs"
CSRC = ROOT / "lbm-arrayfire_b200" / "bindings" / "c_abi_check.c"
LIBDIR = ROOT / "lbm-arrayfire_b200" / "lbm_b200"

C_SCALARS = {"int": "i32", "int32_t": "i32", "int64_t": "i64", "uint32_t": "u32", "uint8_t": "u8",
             "double": "f64", "float": "f32", "size_t": "usize", "void": "void", "char": "char"}
RUST_SCALARS = {"c_int": "i32", "i32": "i32", "i64": "i64", "u32": "u32", "u8": "u8", "c_double": "f64",
                "f64": "f64", "c_float": "f32", "usize": "usize", "c_void": "void", "c_char": "char"}


def c_type(t: str) -> str:
    """Canonical form of a C parameter or return type ('const double* x', 'double out[4]')."""
    t = " ".join(t.split())
    arr = re.search(r"\[\d*\]$", t)
    t = re.sub(r"\s*\w+\s*\[\d*\]$", "*", t) if arr else t
    const = t.startswith("const ")
    t = t[6:] if const else t
    stars = t.count("*")
    base = t.replace("*", " ").split()[0]
    out = C_SCALARS.get(base, base)
    for k in range(stars):
        out = f"{'const' if (const and k == 0) else 'mut'}*{out}"
    return out


def rust_type(t: str) -> str:
    t = " ".join(t.split())
    out_ptrs = []
    while t.startswith("*"):
        kind, t = t[1:].split(" ", 1)
        out_ptrs.append(kind)
    base = RUST_SCALARS.get(t, t)
    for kind in reversed(out_ptrs):
        base = f"{kind}*{base}"
    return base


def header_functions():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    out = {}
    for m in re.finditer(r"^\s*([A-Za-z_][\w\s\*]*?)\b(lbm_\w+)\s*\(([^;]*?)\);", text, flags=re.M | re.S):
        ret, name, params = m.group(1), m.group(2), " ".join(m.group(3).split())
        args = [] if params in ("void", "") else [c_type(re.sub(r"\s*\b\w+$", "", p.strip()) if "[" not in p
                                                         else p.strip()) for p in params.split(",")]
        out[name] = (c_type(ret), args)
    return out


def rust_functions():
    text = RUST.read_text()
    block = text[text.index('extern "C" {'):]
    block = block[:block.index("\n}\n")]
    out = {}
    for m in re.finditer(r"pub fn (lbm_\w+)\((.*?)\)(?:\s*->\s*([^;]+))?;", block, flags=re.S):
        name, params, ret = m.group(1), " ".join(m.group(2).split()), m.group(3)
        args = [rust_type(p.split(":", 1)[1]) for p in params.split(",") if p.strip()] if params else []
        out[name] = (rust_type(ret) if ret else "void", args)
    return out


def test_rust_declares_every_header_function_with_the_same_types():
    h, r = header_functions(), rust_functions()
    assert len(h) >= 50
    assert sorted(h) == sorted(r)
    for name in h:
        assert h[name] == r[name], (name, h[name], r[name])


def struct_fields_c(name):
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    body = re.search(r"typedef struct %s \{(.*?)\} %s;" % (name, name), text, flags=re.S).group(1)
    fields = []
    for decl in body.split(";"):
        decl = " ".join(decl.split())
        if not decl:
            continue
        m = re.match(r"(const )?([\w]+)(\*?) (.*)", decl)
        const, base, ptr, names = m.groups()
        for nm in names.split(","):
            nm = nm.strip()
            arr = re.match(r"(\w+)\[(\w+)\]", nm)
            t = C_SCALARS.get(base, base)
            if ptr:
                t = f"{'const' if const else 'mut'}*{t}"
            if arr:
                fields.append((arr.group(1), f"[{t};{arr.group(2)}]"))
            else:
                fields.append((nm, t))
    return fields


def struct_fields_rust(name):
    body = re.search(r"pub struct %s \{(.*?)\n\}" % name, RUST.read_text(), flags=re.S).group(1)
    fields = []
    for line in body.splitlines():
        m = re.match(r"\s*pub (\w+): (.+),$", line)
        if not m:
            continue
        t = m.group(2).strip()
        arr = re.match(r"\[(.+); (\w+)\]", t)
        fields.append((m.group(1), f"[{rust_type(arr.group(1))};{arr.group(2)}]" if arr else rust_type(t)))
    return fields


@pytest.mark.parametrize("name", ["lbm_cell_class", "lbm_desc"])
def test_rust_structs_mirror_the_header(name):
    c = struct_fields_c(name)
    r = struct_fields_rust(name)
    assert [f for f, _ in c] == [f for f, _ in r]
    for (f, tc), (_, tr) in zip(c, r):
        assert tc == tr, (f, tc, tr)


def build_c_program(tmp_path):
    exe = tmp_path / "c_abi_check"
    out = subprocess.run(["gcc", "-std=c99", "-O2", "-Wall", "-Wextra", "-Werror", "-I", str(ROOT / "include"),
                          str(CSRC), "-L", str(LIBDIR), "-llbm_b200", f"-Wl,-rpath,{LIBDIR}", "-o", str(exe)],
                         capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    return exe


def test_c_layout_equals_the_rust_assertions(tmp_path):
    exe = build_c_program(tmp_path)
    out = subprocess.run([str(exe), "layout"], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0, out.stderr
    c = {}
    for line in out.stdout.splitlines():
        kind, key, val = line.split() if len(line.split()) == 3 else (None, *line.split())
        c[(kind, key)] = int(val)
    rust = RUST.read_text()
    asserted = {}
    for m in re.finditer(r"size_of::<(\w+)>\(\) == (\d+)", rust):
        asserted[("sizeof", m.group(1))] = int(m.group(2))
    for m in re.finditer(r"offset_of!\((\w+), (\w+)\) == (\d+)", rust):
        asserted[("offsetof", f"{m.group(1)}.{m.group(2)}")] = int(m.group(3))
    assert len(asserted) == 2 + 6 + 17
    for key, val in asserted.items():
        assert c[key] == val, (key, c[key], val)
    assert c[(None, "abi_version")] == 1


@pytest.mark.gpu
def test_c_program_steps_a_lattice(tmp_path):
    exe = build_c_program(tmp_path)
    out = subprocess.run([str(exe), "run", "32", "100"], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    line = [ln for ln in out.stdout.splitlines() if ln.startswith("sums ")][0]
    m, jx, jy = (float(v) for v in line.split()[1:])
    assert "steps_done 100" in out.stdout
    p = P.cavity2d(32, 32, 0.1, P.omega_from_re(0.1, 32, 100.0, 0))
    Fo, _, _ = O.run(p, P.rest_state(p), 100)
    so = O.sums(p, Fo)
    assert abs(m - so[0]) / so[0] < 1e-6
    assert np.allclose([jx, jy], so[1:3], rtol=1e-4, atol=1e-6)


def test_rust_constants_match_the_header():
    """Every cell-class flag (#define LBM_CELL_*) and kernel family (enum lbm_kernel) of the header has
    a Rust constant of the same value."""
    import re

    h = HEADER.read_text()
    r = RUST.read_text()
    want = {k: int(v, 0) for k, v in re.findall(r"#define (LBM_CELL_\w+)\s+(0x[0-9a-fA-F]+)u", h)}
    enum = re.search(r"enum lbm_kernel \{([^}]*)\}", h).group(1)
    want.update({k: int(v) for k, v in re.findall(r"(LBM_KERNEL_\w+)\s*=\s*(\d+)", enum)})
    have = {k: int(v, 0) for k, v in re.findall(r"pub const (LBM_(?:CELL|KERNEL)_\w+): \w+ = (0x[0-9a-fA-F]+|\d+);", r)}
    assert len(want) >= 12
    for k, v in want.items():
        assert have.get(k) == v, (k, v, have.get(k))
