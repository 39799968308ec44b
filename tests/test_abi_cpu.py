"""The C ABI without a GPU: the libraries load, export every function the
headers declare, the ctypes mirror has the C struct sizes, the headers build
under -pedantic -Werror as C99/C11/C++11/C++17 and link from C and C++, and the
host-side table validator rejects corrupted tables with the right status."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from bigstickpublick_b200 import _abi, model, engine

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header):
    txt = open(os.path.join(ROOT, "include", header)).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return set(re.findall(r"\b(bsg_\w+)\s*\(", txt)) - {"bsg_tables", "bsg_ctx"}


def exported(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", lib], capture_output=True, text=True).stdout
    return {ln.split()[-1] for ln in out.splitlines() if " T " in ln}


def test_engine_exports_every_declared_symbol():
    path = _abi.lib_path("libbsgpu.so")
    assert os.path.exists(path)
    C.CDLL(path)  # loads without a GPU
    missing = declared("bsg.h") - exported(path)
    assert not missing, missing


def test_host_builder_exports_every_declared_symbol():
    path = _abi.lib_path("libbsghost.so")
    missing = declared("bsg_host.h") - exported(path)
    assert not missing, missing


def test_struct_sizes_match_c(tmp_path):
    src = tmp_path / "sz.c"
    src.write_text('#include "bsg_host.h"\n#include <stdio.h>\nint main(){printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\\n",'
                   'sizeof(bsg_tables),sizeof(bsg_config),sizeof(bsg_lanczos_params),sizeof(bsg_report),'
                   'sizeof(bsg_stats),sizeof(bsg_model_spec),sizeof(bsg_host_tables),sizeof(bsg_tbme),'
                   'sizeof(bsg_tables3),sizeof(bsg_model3_spec));}\n')
    exe = tmp_path / "sz"
    subprocess.check_call(["gcc", "-I" + os.path.join(ROOT, "include"), str(src), "-o", str(exe)])
    c_sizes = [int(x) for x in subprocess.check_output([str(exe)]).split()]
    py = [C.sizeof(s) for s in (_abi.BsgTables, _abi.BsgConfig, _abi.BsgLanczosParams, _abi.BsgReport,
                               _abi.BsgStats, _abi.BsgModelSpec, _abi.BsgHostTables, _abi.BsgTbme,
                               _abi.BsgTables3, _abi.BsgModel3Spec)]
    assert c_sizes == py


@pytest.fixture()
def tables():
    return model.build_tables(model.sd_model(2, 2, seed=1))


def test_validator_accepts_builder_tables(tables):
    assert engine.validate_tables(tables) == (0, "")


@pytest.mark.parametrize("field,index,value,status,needle", [
    ("p1b_isd", 0, 123456789, 2, "pstart"),
    ("p2b_op", 0, 10 ** 6, 2, "hmatpp"),
    ("n1b_phase", 0, 3, 1, "phase"),
    ("n2b_isd", 0, 10 ** 6, 1, "n2b isd/fsd"),
    ("pstart", 1, 0, 1, "pstart"),
    ("hchar", 0, ord("x"), 1, "hchar"),
    ("optype", 0, 99, 1, "optype"),
])
def test_validator_rejects_corrupted_tables(tables, field, index, value, status, needle):
    tables.a[field] = tables.a[field].copy()
    tables.a[field][index] = value
    st, msg = engine.validate_tables(tables)
    assert st == status, (st, msg)
    assert needle in msg


def test_validator_rejects_range_past_array(tables):
    ib = int(np.nonzero(tables.a["optype"] == 4)[0][0])
    tables.a["pxend"] = tables.a["pxend"].copy()
    tables.a["pxend"][ib] = tables.s["np1b"] + 5
    st, msg = engine.validate_tables(tables)
    assert st == 2 and "PN range" in msg


_HOST_PROGRAM = r'''
#include "bsg_host.h"
#include <stdio.h>
#include <string.h>
int main(void) {
    bsg_tables t;
    char msg[256];
    int st;
    memset(&t, 0, sizeof t);
    st = bsg_validate_tables(&t, msg, sizeof msg);
    printf("%d|%s|%s|%d\n", st, msg, bsg_strerror(BSG_ERR_BAD_TABLE), bsg_host_build(NULL, NULL));
    return 0;
}
'''


@pytest.mark.parametrize("lang,std", [("c", "c99"), ("c", "c11"), ("c++", "c++11"), ("c++", "c++17")])
def test_headers_build_strictly_and_link_from_c_and_cpp(tmp_path, lang, std):
    # a C or C++ host includes both headers under -pedantic -Werror and calls
    # host-only entry points through the extern "C" declarations (no GPU call)
    src = tmp_path / ("prog.c" if lang == "c" else "prog.cpp")
    src.write_text(_HOST_PROGRAM)
    exe = tmp_path / "prog"
    pkg = os.path.join(ROOT, "bigstickpublick_b200")
    cc = "gcc" if lang == "c" else "g++"
    r = subprocess.run([cc, "-std=" + std, "-Wall", "-Wextra", "-pedantic", "-Werror",
                        "-I" + os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                        "-L" + pkg, "-lbsgpu", "-lbsghost", "-Wl,-rpath," + pkg],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    st, msg, name, host_st = subprocess.check_output([str(exe)], text=True).strip().split("|")
    assert _abi.STATUS_NAMES[int(st)] == "BSG_ERR_BAD_TABLE" and "empty basis" in msg
    assert name == "table failed validation"
    assert _abi.STATUS_NAMES[int(host_st)] == "BSG_ERR_ARG"   # null output pointer
