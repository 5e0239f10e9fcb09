"""The C-ABI library loads and exports every entry point include/*.h declares
(no compute calls: runs without a GPU)."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

import sgs

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(REPO, "include", "*.h")):
        txt = open(h).read()
        names |= set(re.findall(r"SGS_API\s+[\w\s\*]+?\b(sgs_\w+)\s*\(", txt))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "sgs_create" in names and "sgs_apply_batch" in names
    assert len(names) >= 16


def test_library_exports_every_declared_symbol():
    L = sgs.lib()
    missing = [n for n in declared_symbols() if not hasattr(L, n)]
    assert not missing, missing
    assert set(sgs.EXPORTS) <= set(declared_symbols())


def test_config_defaults_without_gpu():
    c = sgs.default_config()
    assert c.segments == 512 and c.max_rounds == 1000 and c.group_size == 4
    assert abs(c.pr_alpha - 0.85) < 1e-12
    # the documented engine defaults: invalidation and post-sweep rounds and
    # PageRank's pull rounds as cooperative launches; PageRank sweeps as
    # pulls; the reference's re-push repair; warm PageRank starts; an update
    # may restart a served query twice
    assert c.persistent == 14 and c.pull == 1 and c.repair == 0 and c.pr_warm == 1
    assert c.serve_restarts == 2 and c.host_policy == 0 and c.weight_mode == sgs.W_EXPLICIT
    assert sgs.lib().sgs_version().startswith(b"sgs-b200")


def test_create_fails_cleanly_without_gpu():
    """Without a usable GPU, create returns an error code, never exits."""
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        pytest.skip("GPU present")
    with pytest.raises(sgs.SgsError):
        sgs.Engine()


def test_null_arguments_rejected():
    L = sgs.lib()
    assert L.sgs_create(None, None) < 0
    assert L.sgs_apply_batch(None, None, None, None, 0, None, None, 0, 0) < 0
    assert b"null" in L.sgs_last_error()


def test_host_update_generator_matches_oracle():
    """The product's update-stream generator reproduces the oracle's."""
    import oracle as O

    nv, row, col = O.rmat_csr(11, 16, 2)
    a = sgs.gen_update_stream(nv, row, col, 1234, 700, 900)
    b = O.gen_updates(nv, row, col, 1234, 700, 900)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    w = sgs.hash_weights(5, a[0], a[1])
    assert np.array_equal(w, [O.weight_of(5, int(u), int(v)) for u, v in zip(a[0], a[1])])


def _c_layout(struct, fields):
    """sizeof and field offsets of a C struct of include/sgs.h, from a tiny
    program compiled here with the host compiler."""
    import shutil
    import subprocess
    import tempfile

    cc = shutil.which("gcc") or shutil.which("cc")
    if not cc:
        pytest.skip("no C compiler")
    src = ["#include <stdio.h>", "#include <stddef.h>", '#include "sgs.h"', "int main(void) {",
           f'  printf("%zu\\n", sizeof({struct}));']
    src += [f'  printf("%zu\\n", offsetof({struct}, {f}));' for f in fields]
    src += ["  return 0;", "}"]
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "l.c")
        exe = os.path.join(d, "l")
        open(c, "w").write("\n".join(src) + "\n")
        subprocess.check_call([cc, "-std=c99", "-I", os.path.join(REPO, "include"), c, "-o", exe])
        vals = [int(x) for x in subprocess.check_output([exe]).split()]
    return vals[0], vals[1:]


@pytest.mark.parametrize("py, c", [(sgs.Config, "sgs_config"), (sgs.EngineStats, "sgs_engine_stats"),
                                   (sgs.QueryStats, "sgs_query_stats"),
                                   (sgs.KernelStats, "sgs_kernel_stats"), (sgs.Tune, "sgs_tune"),
                                   (sgs.Request, "sgs_request"), (sgs.Completion, "sgs_completion"),
                                   (sgs.PprStats, "sgs_ppr_stats")])
def test_ctypes_structs_match_the_header(py, c):
    """The binding's ctypes mirrors have the C structs' size and field
    offsets, so fields appended to the header cannot drift apart."""
    names = [f for f, _ in py._fields_]
    size, offs = _c_layout(c, names)
    assert ctypes.sizeof(py) == size
    assert [getattr(py, n).offset for n in names] == offs


def test_sample_apps_library_loads_and_exports():
    """The AppBase functor samples (include/sgs_app.cuh instantiated in
    c-gpustreamgraph_b200/apps) build into a library that loads without a GPU
    and exports its drivers."""
    sgs.lib()
    L = ctypes.CDLL(os.path.join(REPO, "c-gpustreamgraph_b200", "lib", "libsgs_apps.so"))
    for n in ("sgs_sample_app_create", "sgs_sample_app_start", "sgs_sample_app_values",
              "sgs_sample_app_parents", "sgs_sample_app_stats", "sgs_sample_app_destroy",
              "sgs_sample_refstyle_sssp"):
        assert hasattr(L, n), n
    # without a graph (or a GPU) an attach is refused with a status, not a crash
    L.sgs_sample_app_create.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_uint32, ctypes.c_double,
                                        ctypes.c_double, ctypes.POINTER(ctypes.c_void_p)]
    assert L.sgs_sample_app_create(None, 1, 0, 0.0, 0.85, None) < 0
