"""CPU: the C-ABI libraries load, and export every function their headers declare.

No compute runs here (no GPU in this suite): only symbol resolution and the
host-side argument checks that return before touching a device.
"""
import ctypes
import os
import re

import pytest

import casgemm

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", h) for h in ("casgemm.h", "casgemm_data.h")]
DECL = re.compile(r"^[A-Za-z_][\w \t\*]*?\b(cas_\w+)\s*\(", re.M)


def declared(path):
    text = open(path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(DECL.findall(text)))


@pytest.mark.parametrize("header", HEADERS, ids=os.path.basename)
def test_every_declared_symbol_is_exported(header):
    lib = casgemm.load()
    names = declared(header)
    assert len(names) >= 8
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, f"not exported: {missing}"


def test_expected_entry_points_declared():
    names = set(declared(HEADERS[0]))
    for n in ("cas_create", "cas_destroy", "cas_spgemm", "cas_flp_populate", "cas_scan", "cas_hash_symb",
              "cas_hash_numc", "cas_hsersc_numc", "cas_hybacc_numc", "cas_csr_free", "cas_scan_noalloc",
              "cas_csr_transpose", "cas_serve_submit"):
        assert n in names


def test_host_argument_checks_need_no_device():
    lib = casgemm.load()
    # NULL context / outputs are rejected before any CUDA call
    assert lib.cas_spgemm(None, 2, None, None, None, None) == 1
    assert lib.cas_scan(None, None, None, 4) == 1
    fn = lib.cas_scan_noalloc
    fn.restype = ctypes.c_int32
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p]
    assert fn(None, None, 5, None) == 1
    assert fn(ctypes.c_void_p(16), ctypes.c_void_p(16), 16384 * 4096 + 1, None) == 7


def test_oracle_library_exports():
    import oracle
    lib = oracle.oracle_lib()
    for n in ("orc_flp_populate", "orc_scan", "orc_hash_symb", "orc_spgemm", "orc_radix_sort_kv",
              "orc_pack_morsels", "orc_sort_rows", "orc_intprod"):
        assert hasattr(lib, n)


def test_autotuner_key_is_a_function_of_the_degrees():
    A = casgemm.gen_er(10, 32, 1)
    G = casgemm.gen_g500(12, 8, 1)
    assert casgemm.Autotuner.key(A, A) == casgemm.Autotuner.key(casgemm.gen_er(10, 32, 9), casgemm.gen_er(10, 32, 9))
    assert casgemm.Autotuner.key(A, A) != casgemm.Autotuner.key(G, G)
    assert casgemm.Autotuner.key(A, A).endswith("_f64")


# every struct of include/casgemm.h that casgemm.py mirrors with ctypes
MIRRORS = {"cas_csr": "CasCsr", "cas_runtime": "CasRuntime", "cas_stats": "CasStats", "cas_job": "CasJob",
           "cas_batch_stats": "CasBatchStats", "cas_server_opts": "CasServerOpts", "cas_result": "CasResult",
           "cas_server_stats": "CasServerStats", "cas_tuning": "CasTuning"}


def test_ctypes_mirrors_match_the_header(tmp_path):
    """Size and every field's offset of each mirrored struct, as the C compiler lays them out."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "casgemm.h"', "int main(void) {"]
    for c_name, py_name in MIRRORS.items():
        lines.append(f'printf("{c_name} size %zu\\n", sizeof({c_name}));')
        for f, _ in getattr(casgemm, py_name)._fields_:
            lines.append(f'printf("{c_name} {f} %zu\\n", offsetof({c_name}, {f}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", os.path.join(ROOT, "include"), "-o", str(exe), str(src)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {}
    for ln in out:
        if ln:
            s, f, v = ln.split()
            got[(s, f)] = int(v)
    for c_name, py_name in MIRRORS.items():
        cls = getattr(casgemm, py_name)
        assert ctypes.sizeof(cls) == got[(c_name, "size")], c_name
        for f, _ in cls._fields_:
            assert getattr(cls, f).offset == got[(c_name, f)], (c_name, f)
