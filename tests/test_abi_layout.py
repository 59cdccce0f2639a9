"""The Python bindings' ctypes structures match include/svf.h field by field:
a small C program compiled against the header prints sizeof and offsetof of
every field, and the ctypes layouts must agree (a mismatch would hand the
library shifted options silently).  The host-only defaults of the option
structures are checked too.  No GPU is needed."""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

import tempestrenderer_b200 as svf

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# C struct name -> ctypes class
STRUCTS = {
    "svf_lsq_options": svf.LsqOptions,
    "svf_texel_stats": svf.TexelStats,
    "svf_layout_desc": svf.LayoutDesc,
    "svf_btf_view": svf.BtfView,
    "svf_fit_options": svf.FitOptions,
    "svf_btf_info": svf.BtfInfo,
    "svf_svbrdf_maps": svf.SvbrdfMaps,
    "svf_mlp_train_options": svf.MlpTrainOptions,
    "svf_maps": svf.Maps,
    "svf_run_stats": svf.RunStats,
}


@pytest.fixture(scope="module")
def c_layout(tmp_path_factory):
    cc = shutil.which("gcc") or shutil.which("cc")
    if not cc:
        pytest.skip("no C compiler")
    d = tmp_path_factory.mktemp("abi")
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "svf.h"', "int main(void) {"]
    for cname, cls in STRUCTS.items():
        lines.append(f'printf("{cname} sizeof %zu\\n", sizeof({cname}));')
        for fname, _ in cls._fields_:
            lines.append(f'printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["return 0;", "}"]
    src, exe = d / "layout.c", d / "layout"
    src.write_text("\n".join(lines))
    subprocess.run([cc, "-std=c11", "-I", os.path.join(REPO, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    table = {}
    for line in out.splitlines():
        cname, fname, value = line.split()
        table[(cname, fname)] = int(value)
    return table


@pytest.mark.parametrize("cname", sorted(STRUCTS))
def test_ctypes_layout_matches_the_header(c_layout, cname):
    cls = STRUCTS[cname]
    assert C.sizeof(cls) == c_layout[(cname, "sizeof")], cname
    for fname, _ in cls._fields_:
        assert getattr(cls, fname).offset == c_layout[(cname, fname)], (cname, fname)


def test_option_defaults(svf_lib):
    o = svf.MlpTrainOptions()
    svf_lib.svf_mlp_train_options_default(C.byref(o))
    assert (o.texels, o.epochs, o.batch, o.max_iterations, o.features) == (1 << 20, 48, 4096, 1024,
                                                                          svf.SVF_MLP_FEATURES_BINS)
    assert o.lr == pytest.approx(2e-3)
    lo = svf.LsqOptions()
    svf_lib.svf_lsq_options_default(C.byref(lo))
    assert lo.restarts == 1 and lo.mse_target == 1e-6
    # the reference's BreakOnSmallStep is a float 1e-3, widened
    assert lo.break_on_small_step == float(np.float32(1e-3))
