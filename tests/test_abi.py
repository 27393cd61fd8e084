"""The C ABI: include/mcg.h, the built library and the Python mirror agree.

No compute call is made here (no GPU is needed): the library must load, export
every function the header declares, and the ctypes structures must have the C
compiler's sizes and field offsets.
"""
import ctypes as C
import os
import re
import subprocess
import tempfile

import pytest

import helpers as H
from rust_pricing_b200 import _abi as A
from rust_pricing_b200 import _native

HEADER = os.path.join(H.ROOT, "include", "mcg.h")


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:mcg_status|uint32_t|const char\*|void)\s+(mcg_\w+)\s*\(", text, re.M)))


def test_header_declares_the_entry_points():
    names = declared_functions()
    assert set(names) == set(_native.EXPORTS)


def test_library_loads_and_exports_every_declared_symbol():
    lib = _native.library()
    for name in declared_functions():
        assert hasattr(lib, name), name
    assert lib.mcg_abi_version() == A.ABI_VERSION


def test_build_recipe_targets_sm_100a():
    import build as recipe
    assert recipe.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]


STRUCTS = {
    "mcg_curve": A.Curve, "mcg_local_variance_grid": A.LocalVarianceGrid,
    "mcg_product_desc": A.ProductDesc, "mcg_plan_desc": A.PlanDesc, "mcg_statistics": A.Statistics,
    "mcg_estimate": A.Estimate, "mcg_product_result": A.ProductResult,
    "mcg_error_record": A.ErrorRecord, "mcg_result": A.Result,
    "mcg_lsm_desc": A.LsmDesc, "mcg_lsm_date_model": A.LsmDateModel, "mcg_lsm_result": A.LsmResult,
    "mcg_book_options": A.BookOptions, "mcg_book_report": A.BookReport, "mcg_surface_desc": A.SurfaceDesc,
    "mcg_vega_kt_basis": A.VegaKtBasis, "mcg_vega_kt_projection": A.VegaKtProjection,
    "mcg_dual_desc": A.DualDesc, "mcg_dual_result": A.DualResult, "mcg_dividends": A.Dividends,
    "mcg_asset_desc": A.AssetDesc, "mcg_multi_asset_desc": A.MultiAssetDesc,
    "mcg_multi_asset_result": A.MultiAssetResult, "mcg_bump_request": A.BumpRequest,
    "mcg_bump_estimate": A.BumpEstimate, "mcg_bump_report": A.BumpReport,
}


def test_ctypes_layout_matches_c_compiler():
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void){"]
    for cname, cls in STRUCTS.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for field, _ in cls._fields_:
            # a trailing underscore keeps a C name that is a Python keyword (lambda)
            lines.append(f'printf("{cname}.{field} %zu\\n", offsetof({cname}, {field.rstrip("_")}));')
    lines.append("return 0;}")
    with tempfile.TemporaryDirectory() as d:
        src, exe = os.path.join(d, "layout.c"), os.path.join(d, "layout")
        open(src, "w").write("\n".join(lines))
        subprocess.run(["gcc", "-std=c11", src, "-o", exe], check=True)
        got = dict(line.split() for line in subprocess.run([exe], capture_output=True, text=True).stdout.splitlines())
    for cname, cls in STRUCTS.items():
        assert int(got[cname]) == C.sizeof(cls), cname
        for field, _ in cls._fields_:
            assert int(got[f"{cname}.{field}"]) == getattr(cls, field).offset, f"{cname}.{field}"


def test_no_device_means_a_loud_error_not_a_fallback():
    """Without a visible GPU, plan creation fails with MCG_ERR_CUDA."""
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is visible")
    except ImportError:
        pass
    from rust_pricing_b200 import workloads as W
    with pytest.raises(_native.EngineError) as err:
        _native.Plan(W.european_bs(paths=1024))
    assert err.value.name == "cuda"
