"""The C ABI library loads on a CPU-only host and exports every symbol that
include/tagmatch_b200.h declares; host-only calls work without a GPU."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from tagmatch_b200 import _native, build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "tagmatch_b200.h")


def declared_symbols():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(tm_[a-z_0-9]+)\s*\(", src)) - {"tm_match_callback"})


def test_header_symbols_exported():
    lib = ctypes.CDLL(build.LIB)
    syms = declared_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(lib, s), s
    # and the Python binding covers every one of them
    assert sorted(_native.SIGNATURES) == syms


def test_status_codes_match_header():
    src = open(HEADER).read()
    for name in ["TM_OK", "TM_ERR_INVALID", "TM_ERR_CUDA", "TM_ERR_STATE", "TM_ERR_CAPACITY", "TM_ERR_NOMEM",
                 "TM_ERR_IO", "TM_ERR_TIMEOUT", "TM_ERR_INTERNAL"]:
        m = re.search(r"#define " + name + r" \(?(-?\d+)\)?", src)
        assert int(m.group(1)) == getattr(_native, name)


def test_host_only_calls_without_gpu():
    lib = _native.load()
    h = ctypes.c_void_p()
    assert lib.tm_create(ctypes.byref(h)) == 0
    w = np.arange(6, dtype=np.uint32)
    k = np.array([1, 2], dtype=np.uint32)
    p32 = lambda a: a.ctypes.data_as(_native.u32p)  # noqa: E731
    assert lib.tm_add(h, p32(w), p32(k), 2) == 0
    assert lib.tm_remove(h, p32(w), 1) == 0
    assert lib.tm_set_latency_limit_ms(h, 250) == 0
    assert lib.tm_get_latency_limit_ms(h) == 250
    assert lib.tm_set_database_filename(h, b"/tmp/x.db") == 0
    assert lib.tm_get_database_filename(h) == b"/tmp/x.db"
    assert lib.tm_set_batch_limit(h, 0) == _native.TM_ERR_INVALID
    assert lib.tm_add(None, p32(w), p32(k), 2) == _native.TM_ERR_INVALID
    assert lib.tm_consolidate(h, 0, 1) == _native.TM_ERR_INVALID
    assert b"partition size" in lib.tm_last_error(h)
    assert lib.tm_version().startswith(b"tagmatch-b200")
    lib.tm_destroy(h)


def test_facade_headers_compile_and_bitvector_semantics(tmp_path):
    """The tagmatch.hh-compatible headers compile; bitvector<192> agrees with
    the reference's layout and order on random vectors (CPU only)."""
    src = tmp_path / "bv.cc"
    src.write_text(r'''
#include <cstdio>
#include <cstdlib>
#include <sstream>
#include "tagmatch.hh"
#include "synchronous_match_handler.hh"
int main() {
    srand(7);
    int bad = 0;
    for (int t = 0; t < 20000; ++t) {
        std::string a(192, '0'), b(192, '0');
        for (int i = 0; i < 192; ++i) { if (rand() % 5 == 0) a[i] = '1'; if (rand() % 2 == 0) b[i] = '1'; }
        if (t % 3 == 0) b = a;
        filter_t x(a), y(b);
        bool sub = true;
        for (int i = 0; i < 192; ++i) if (a[i] == '1' && b[i] == '0') sub = false;
        if (x.subset_of(y) != sub) ++bad;
        // order: first differing character decides, '1' is greater
        int d = 0; while (d < 192 && a[d] == b[d]) ++d;
        bool lt = d < 192 && b[d] == '1';
        if ((x < y) != lt) ++bad;
        if (d < 192 && (int)x.leftmost_diff(y) != d) ++bad;
        std::ostringstream os; x.write_ascii(os); if (os.str() != a) ++bad;
        std::ostringstream bo; x.write_binary(bo);
        std::istringstream bi(bo.str()); filter_t z; z.read_binary(bi); if (!(z == x)) ++bad;
        unsigned pc = 0; for (char c : a) pc += c == '1'; if (x.popcount() != pc) ++bad;
        unsigned nb = x.next_bit(0), first = 0; while (first < 192 && a[first] != '1') ++first;
        if (nb != first) ++bad;
        for (unsigned r = 0; r <= 192; r += 37) {
            bool ps = true; for (unsigned i = 0; i < r; ++i) if (a[i] == '1' && b[i] == '0') ps = false;
            if (x.prefix_subset_of(y, r) != ps) ++bad;
        }
    }
    std::printf("%d\n", bad);
    return bad != 0;
}
''')
    exe = tmp_path / "bv"
    inc = os.path.join(ROOT, "include", "tagmatch")
    subprocess.check_call(["g++", "-O1", "-std=c++17", "-I" + inc, str(src), "-o", str(exe)])
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr


def header_structs():
    """name -> [(C type, field)] for every `typedef struct { ... } name;` in the header."""
    src = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    out = {}
    for body, name in re.findall(r"typedef struct \{(.*?)\}\s*(\w+);", src, flags=re.S):
        fields = []
        for decl in body.split(";"):
            decl = decl.strip()
            if not decl:
                continue
            ctype, names = decl.split(None, 1)
            fields += [(ctype, n.strip()) for n in names.split(",")]
        out[name] = fields
    return out


def test_struct_layouts_match_header(tmp_path):
    """The ctypes mirrors of the header's structs have the same fields, types
    and order, and the same size as the C compiler gives them."""
    ctypes_of = {"uint64_t": ctypes.c_uint64, "uint32_t": ctypes.c_uint32, "double": ctypes.c_double}
    mirrors = {"tm_table_info": _native.TableInfo, "tm_match_stats": _native.MatchStats}
    structs = header_structs()
    assert set(mirrors) <= set(structs)
    for cname, mirror in mirrors.items():
        assert [(ctypes_of[t], n) for t, n in structs[cname]] == [(t, n) for n, t in mirror._fields_], cname
    prog = tmp_path / "sizes.c"
    prog.write_text('#include <stdio.h>\n#include "tagmatch_b200.h"\n'
                    'int main(void) { printf("%zu %zu\\n", sizeof(tm_table_info), sizeof(tm_match_stats)); return 0; }\n')
    exe = tmp_path / "sizes"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), "-o", str(exe), str(prog)], check=True)
    sizes = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    assert sizes == [ctypes.sizeof(_native.TableInfo), ctypes.sizeof(_native.MatchStats)]
