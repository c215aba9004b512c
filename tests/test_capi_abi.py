"""The product library loads and exports exactly what include/*.h declares.

No GPU needed: only symbol resolution and argument validation that returns
before any CUDA call.
"""
import ctypes as C
import os
import re
import subprocess

import pytest

from gasal_b200 import lib as gl

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "include")


@pytest.fixture(scope="module")
def so():
    if not os.path.exists(gl.LIB_PATH):
        gl.build()
    return gl.lib()


def c_abi_names():
    txt = open(os.path.join(INC, "gasal_b200_capi.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b((?:gasal_c|gb)_[a-z0-9_]+)\s*\(", txt)))


def test_every_c_abi_symbol_exported(so):
    names = c_abi_names()
    assert len(names) >= 20
    for n in names:
        assert hasattr(so, n), f"{n} declared in gasal_b200_capi.h but not exported"
    # the Python binding declares a signature for every exported entry point
    assert set(names) == set(gl.SIGNATURES), set(names) ^ set(gl.SIGNATURES)


CXX_API = ["gasal_copy_subst_scores", "gasal_aln_async", "gasal_is_aln_async_done", "gasal_init_gpu_storage_v",
           "gasal_init_streams", "gasal_destroy_streams", "gasal_destroy_gpu_storage_v", "gasal_gpu_mem_alloc",
           "gasal_gpu_mem_free", "gasal_host_batch_new", "gasal_host_batch_destroy", "gasal_host_batch_getlast",
           "gasal_host_batch_reset", "gasal_host_batch_fill", "gasal_host_batch_add", "gasal_host_batch_addbase",
           "gasal_host_batch_print", "gasal_host_batch_printall", "gasal_host_alns_resize", "gasal_op_fill",
           "gasal_set_device", "gasal_res_new_host", "gasal_res_new_device", "gasal_res_new_device_cpy",
           "gasal_res_destroy_host", "gasal_res_destroy_device", "Parameters::Parameters", "Parameters::parse",
           "Parameters::print", "Parameters::help", "Parameters::failure", "Parameters::fileopen"]


def test_cxx_drop_in_symbols(so):
    """GASAL2's C++ entry points (reference src/ctors.h, host_batch.h,
    interfaces.h, res.h, gasal_align.h, args_parser.h) exist with C++ linkage."""
    out = subprocess.run(["nm", "-DC", "--defined-only", gl.LIB_PATH], capture_output=True, text=True).stdout
    for name in CXX_API:
        assert re.search(r"\b" + re.escape(name) + r"\(", out), f"{name} missing"
    # signatures the reference declares (spot checks of argument lists)
    assert "gasal_aln_async(gasal_gpu_storage_t*, unsigned int, unsigned int, unsigned int, Parameters*)" in out
    assert "gasal_host_batch_fill(gasal_gpu_storage_t*, unsigned int, char const*, unsigned int, data_source)" in out
    assert "gasal_init_streams(gasal_gpu_storage_v*, int, int, int, Parameters*)" in out


def test_struct_layouts_match_reference_abi():
    """The drop-in header keeps the reference's struct layouts (sizes and
    member offsets of gasal_gpu_storage_t, gasal_res_t, host_batch_t)."""
    src = r'''
#include <cstddef>
#include <cstdio>
#include "gasal.h"
int main() {
  printf("%zu %zu %zu %zu %zu %zu %zu %zu\n", sizeof(gasal_gpu_storage_t), offsetof(gasal_gpu_storage_t, host_res),
         offsetof(gasal_gpu_storage_t, packed_tb_matrices), offsetof(gasal_gpu_storage_t, str),
         sizeof(gasal_res_t), offsetof(gasal_res_t, n_cigar_ops), sizeof(host_batch_t), sizeof(gasal_subst_scores));
}
'''
    import tempfile
    d = tempfile.mkdtemp()
    open(os.path.join(d, "l.cpp"), "w").write(src)
    subprocess.run(["/usr/bin/g++", "-I", INC, "-I/usr/local/cuda/include", os.path.join(d, "l.cpp"), "-o",
                    os.path.join(d, "l")], check=True)
    got = subprocess.run([os.path.join(d, "l")], capture_output=True, text=True).stdout.split()
    # The same program compiled against the reference's own src/gasal.h (its
    # CUDA include path pointed at this toolkit) prints these numbers on LP64.
    assert got == ["272", "160", "248", "256", "56", "48", "32", "16"], got


def test_argument_errors_return_status(so):
    """Bad arguments come back as GB_ERR_ARG, no process exit."""
    assert so.gasal_c_params_set(None, None) == -1
    assert so.gasal_c_aln_async(None, 8, 8, 1, None) == -1
    assert so.gasal_c_is_aln_async_done(None) == -1
    assert so.gasal_c_init_streams(None, 8, 8, 1, None) == -1
    assert so.gb_set_reference_max_query_len(0) == -1
    assert so.gb_set_tb_budget_mb(0) == -1
    p = so.gasal_c_params_new()
    assert p
    so.gasal_c_params_free(p)


def test_product_fails_loudly_without_library(monkeypatch):
    monkeypatch.setattr(gl, "_lib", None)
    monkeypatch.setattr(gl, "LIB_PATH", "/nonexistent/libgasal_b200.so")
    with pytest.raises(gl.GasalError):
        gl.lib()


def test_tuning_and_graph_settings_validate(so):
    """Launch tuning round-trips and rejects values the kernels cannot take
    (no GPU needed: these only change library settings)."""
    from gasal_b200.lib import GbTuning
    import ctypes as C
    cur = GbTuning()
    assert so.gb_get_tuning(C.byref(cur)) == 0
    for bad in (GbTuning(256, 32, 0, 1, 1, 1, 16), GbTuning(64, 4, 0, 1, 1, 1, 16), GbTuning(64, 32, -1, 1, 1, 1, 16),
                GbTuning(64, 32, 0, 1, 1, 1, 4), GbTuning(64, 32, 0, 1, 1, 1, 24), GbTuning(64, 32, 0, 1, 1, 1, 128)):
        assert so.gb_set_tuning(C.byref(bad)) == -1
    ok = GbTuning(128, 48, 4096, 0, 0, 0, 8)
    assert so.gb_set_tuning(C.byref(ok)) == 0
    back = GbTuning()
    so.gb_get_tuning(C.byref(back))
    assert (back.block, back.wc_min_qregs, back.min_order_pairs, back.ksw_warp, back.split_start,
            back.persistent, back.wc_group) == (128, 48, 4096, 0, 0, 0, 8)
    assert so.gb_set_tuning(C.byref(cur)) == 0
    assert so.gb_set_graphs(0) == 0 and so.gb_set_graphs(1) == 0
    counts = (C.c_int64 * 4)()
    assert so.gb_graph_stats(counts) == 0
