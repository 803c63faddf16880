"""The C-ABI library loads and exports every symbol include/glc.h declares, and argument checks
that need no device answer on CPU."""
import ctypes as C
import os
import re

from conftest import ROOT, load_package

HEADER = os.path.join(ROOT, "include", "glc.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(glc_[a-z0-9_]+)\s*\(", text)))


def test_every_declared_symbol_is_exported():
    g = load_package()
    lib = C.CDLL(g.LIB_PATH)
    names = declared_functions()
    assert len(names) > 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_the_header():
    g = load_package()
    bound = set(g._lib.SIGNATURES) | {"glc_server_create", "glc_server_submit", "glc_server_cancel", "glc_server_wait",
                                      "glc_server_release", "glc_server_get_stats", "glc_server_destroy"}
    assert set(declared_functions()) <= bound


def test_contract_checks_without_a_device():
    g = load_package()
    L = g._lib.lib()
    # log_n = 0 is rejected before any device call (ntt.rs:192)
    assert L.glc_batch_ntt_in_place(None, 64, 0, 1, 0, 64, False, False, 0, 0, None) == 1
    assert b"log_n" in L.glc_last_error_message()
    # offset + n > stride (ntt.rs:350)
    assert L.glc_batch_ntt_in_place(None, 64, 6, 1, 1, 64, False, False, 0, 0, None) == 1
    # results_len not a multiple of 4 (poseidon2.rs:190)
    assert L.glc_poseidon2_compute_leaf_hashes(None, 16, None, 6, 0, False, False, None) == 1
    assert L.glc_poseidon2_compute_node_hashes(None, 16, None, 4, None) == 1
    assert L.glc_bit_reverse(None, 8, None, 8, 6, 1, None) == 1  # rows not a power of two
    assert L.glc_tuning_set_p2(None) == 1


def test_header_compiles_as_c_and_links(tmp_path):
    # a C11 caller (the Rust FFI and cgo-style bindings see the same declarations) compiles
    # against include/glc.h, links libglc.so and gets a contract violation back without a device
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        import pytest
        pytest.skip("no C compiler")
    g = load_package()
    src = tmp_path / "caller.c"
    src.write_text(
        '#include <stdio.h>\n#include <string.h>\n#include "glc.h"\n'
        "int main(void) {\n"
        "  glc_status s = glc_batch_ntt_in_place(NULL, 64, 0, 1, 0, 64, false, false, 0, 0, NULL);\n"
        '  if (s != 1 || !strstr(glc_last_error_message(), "log_n")) return 1;\n'
        '  printf("ok\\n");\n  return 0;\n}\n')
    exe = tmp_path / "caller"
    libdir = os.path.dirname(g.LIB_PATH)
    r = subprocess.run([cc, "-std=c11", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
                        str(src), "-o", str(exe), "-L", libdir, "-lglc", "-Wl,-rpath," + libdir],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and r.stdout.strip() == "ok", (r.returncode, r.stdout, r.stderr)


def test_round_constants_query_without_a_device():
    """The installed-constants query is host bookkeeping: it answers without a GPU, and a process
    that never called glc_poseidon2_set_round_constants reports the placeholder set."""
    g = load_package()
    assert g.poseidon2.round_constants_installed() is False
    L = g._lib.lib()
    assert L.glc_poseidon2_round_constants_installed(None) == 1
