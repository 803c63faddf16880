"""The Rust bindings (zksync-crypto-gpu_b200/rust/, not compiled here: no Rust toolchain) declare
libglc's functions exactly as include/glc.h does: glc-sys covers every function with the same
name and argument count, and boojum-cuda-glc's typed block declares only functions of the header,
each with the header's argument count.  The library itself exports every declared symbol."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
RUST = os.path.join(ROOT, "zksync-crypto-gpu_b200", "rust")


def split_args(text):
    text = text.strip()
    if text in ("", "void"):
        return []
    depth, cur, out = 0, "", []
    for ch in text:
        if ch in "(<[":
            depth += 1
        elif ch in ")>]":
            depth -= 1
        if ch == "," and depth == 0:
            out.append(cur)
            cur = ""
        else:
            cur += ch
    if cur.strip():
        out.append(cur)
    return [a.strip() for a in out if a.strip()]


def header_functions():
    src = open(os.path.join(ROOT, "include", "glc.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    out = {}
    for m in re.finditer(r"\b(glc_\w+)\s*\(([^;{]*?)\)\s*;", src, flags=re.S):
        out[m.group(1)] = len(split_args(m.group(2)))
    return out


def rust_extern_functions(path):
    src = open(path).read()
    src = re.sub(r"//[^\n]*", "", src)
    out = {}
    for block in re.finditer(r'extern\s+"C"\s*\{(.*?)\n\s*\}', src, flags=re.S):
        for m in re.finditer(r"pub\s+fn\s+(glc_\w+)\s*\((.*?)\)\s*(->[^;]*)?;", block.group(1), flags=re.S):
            out[m.group(1)] = len(split_args(m.group(2)))
    return out


def test_header_parses():
    h = header_functions()
    assert len(h) >= 40
    assert h["glc_batch_ntt_out_of_place"] == 15 and h["glc_launch_count"] == 0


def test_glc_sys_declares_every_header_function():
    h = header_functions()
    r = rust_extern_functions(os.path.join(RUST, "glc-sys", "src", "lib.rs"))
    assert set(r) == set(h), (set(h) - set(r), set(r) - set(h))
    assert all(r[k] == h[k] for k in h), {k: (h[k], r[k]) for k in h if r[k] != h[k]}


def test_boojum_shim_declarations_match_header():
    h = header_functions()
    r = rust_extern_functions(os.path.join(RUST, "boojum-cuda-glc", "src", "lib.rs"))
    assert len(r) >= 14
    assert set(r) <= set(h), set(r) - set(h)
    assert all(r[k] == h[k] for k in r), {k: (h[k], r[k]) for k in r if r[k] != h[k]}


def test_library_exports_every_header_function():
    lib_path = os.path.join(ROOT, "zksync-crypto-gpu_b200", "_build", "libglc.so")
    if not os.path.exists(lib_path):
        import importlib.util
        spec = importlib.util.spec_from_file_location("_glc_build", os.path.join(ROOT, "zksync-crypto-gpu_b200", "build.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        mod.build()
    lib = ctypes.CDLL(lib_path)
    missing = [k for k in header_functions() if not hasattr(lib, k)]
    assert not missing, missing
