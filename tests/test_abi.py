"""CPU: the C-ABI library loads, exports every entry point the header
declares, and its Python mirror agrees with the header's struct layouts and
defaults.  No GPU needed (no compute calls)."""
import ctypes
import os
import re
import subprocess
import tempfile

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
HEADER = os.path.join(REPO, "include", "pincflow_poisson.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(pcf_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol(pcf):
    lib = pcf.load()
    names = declared_functions()
    assert len(names) >= 18
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # nm view of the shared object, independent of ctypes
    out = subprocess.run(["nm", "-D", "--defined-only", pcf._lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (pcf_\w+)", out))
    assert set(names) <= exported, set(names) - exported


def test_bounds_checked_library_exports_the_same_symbols():
    """The -DPCF_BOUNDS_CHECK build (build.py --checked) is a drop-in
    replacement of the library: same declared entry points."""
    path = os.path.join(REPO, "pincflow.jl_b200", "lib", "libpincflow_poisson_checked.so")
    if not os.path.exists(path):
        pytest.skip("checked library not built")
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (pcf_\w+)", out))
    names = declared_functions()
    assert set(names) <= exported, set(names) - exported


def _c_layout():
    code = r"""
#include <stdio.h>
#include <stddef.h>
#include "pincflow_poisson.h"
#define F(T, m) printf(#T "." #m " %zu\n", offsetof(T, m));
int main(void) {
  printf("pcf_dims %zu\npcf_params %zu\npcf_result %zu\n", sizeof(pcf_dims), sizeof(pcf_params), sizeof(pcf_result));
  F(pcf_params, dtau) F(pcf_params, inner_tolerance) F(pcf_params, check_interval)
  F(pcf_params, mg_dtau) F(pcf_params, mg_min_columns) F(pcf_params, mg_operator_bf16)
  F(pcf_params, mg_fused_coarse) F(pcf_params, mg_smoother_fp8)
  F(pcf_result, residual) F(pcf_result, ms_total) F(pcf_dims, device)
  return 0;
}
"""
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "l.c")
        exe = os.path.join(d, "l")
        open(c, "w").write(code)
        subprocess.run(["gcc", "-I", os.path.dirname(HEADER), c, "-o", exe], check=True)
        lines = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split("\n")
    return {ln.split()[0]: int(ln.split()[1]) for ln in lines if ln.strip()}


def test_struct_layouts_match_header(pcf):
    L = pcf._lib
    c = _c_layout()
    assert ctypes.sizeof(L.PcfDims) == c["pcf_dims"]
    assert ctypes.sizeof(L.PcfParams) == c["pcf_params"]
    assert ctypes.sizeof(L.PcfResult) == c["pcf_result"]
    assert L.PcfParams.dtau.offset == c["pcf_params.dtau"]
    assert L.PcfParams.inner_tolerance.offset == c["pcf_params.inner_tolerance"]
    assert L.PcfParams.check_interval.offset == c["pcf_params.check_interval"]
    assert L.PcfParams.mg_dtau.offset == c["pcf_params.mg_dtau"]
    assert L.PcfParams.mg_min_columns.offset == c["pcf_params.mg_min_columns"]
    assert L.PcfParams.mg_operator_bf16.offset == c["pcf_params.mg_operator_bf16"]
    assert L.PcfParams.mg_fused_coarse.offset == c["pcf_params.mg_fused_coarse"]
    assert L.PcfParams.mg_smoother_fp8.offset == c["pcf_params.mg_smoother_fp8"]
    assert L.PcfResult.residual.offset == c["pcf_result.residual"]
    assert L.PcfResult.ms_total.offset == c["pcf_result.ms_total"]
    assert L.PcfDims.device.offset == c["pcf_dims.device"]


def test_params_default_mirror_poisson_namelist(pcf):
    p = pcf._lib.PcfParams()
    assert pcf.load().pcf_params_default(ctypes.byref(p)) == 0
    # PoissonNamelist.jl:48-56
    assert p.tolerance == 1e-8 and p.poisson_iterations == 1000 and p.preconditioner == 1
    assert p.dtau == 1.0 and p.preconditioner_iterations == 2 and p.tolerance_is_relative == 0
    assert p.damp_horizontal_wind_on_rhs == 0 and p.precision == 0 and p.residual == 0 and p.learned == 0
    assert p.multigrid == 0 and p.mg_fused_coarse == -1  # the fused coarse cycle: ensembles only
    nl = pcf.PoissonNamelist().to_c()
    for name, _ in pcf._lib.PcfParams._fields_:
        assert getattr(nl, name) == getattr(p, name), name


def test_error_codes_and_null_arguments(pcf):
    lib = pcf.load()
    assert lib.pcf_strerror(0) == b"success"
    assert b"invalid" in lib.pcf_strerror(-1)
    assert lib.pcf_create(None, None) == pcf._lib.PCF_EINVAL
    assert lib.pcf_params_default(None) == pcf._lib.PCF_EINVAL
    assert lib.pcf_destroy(None) == 0
    assert lib.pcf_solve(None, None, None, None, None, 1.0, 1.0, 1.0, None, None, None) == pcf._lib.PCF_EINVAL
    assert lib.pcf_profile_read(None, 0, None, None, None) == pcf._lib.PCF_EINVAL
    assert lib.pcf_launch_count(None) == 0


def test_create_rejects_bad_dims_before_touching_a_device(pcf):
    lib = pcf.load()
    h = ctypes.c_void_p()
    for dims in [(8, 8, 3, 3, 3, 3, 0, 0), (0, 8, 8, 3, 3, 3, 0, 0), (8, 8, 8, 3, 3, 1, 0, 0),
                 (8, 8, 8, 3, 3, 3, 7, 0)]:
        d = pcf._lib.PcfDims(*dims)
        assert lib.pcf_create(ctypes.byref(h), ctypes.byref(d)) == pcf._lib.PCF_EINVAL


def test_no_device_is_an_error_not_a_fallback(pcf):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    with pytest.raises(pcf.PoissonError) as e:
        pcf.PoissonSolver(pcf.fields.Domain(8, 8, 8))
    assert e.value.code == pcf._lib.PCF_ENODEVICE


def _c_struct_fields(name):
    src = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    body = re.search(r"typedef struct \{([^{}]*)\}\s*" + name + r";", src).group(1)
    fields = []
    for decl in body.split(";"):
        decl = decl.strip()
        if not decl:
            continue
        typ, names = decl.split(None, 1)
        fields += [(n.strip(), typ) for n in names.split(",")]
    return fields


JL_PKG = os.path.join(REPO, "pincflow.jl_b200", "julia", "PinCFlowGPU")
JL_CORE = os.path.join(JL_PKG, "src", "PinCFlowGPU.jl")
JL_EXT = os.path.join(JL_PKG, "ext", "PinCFlowGPUExt.jl")


def _julia_struct_fields(name):
    src = open(JL_CORE).read()
    body = re.search(r"(?:mutable )?struct " + name + r"\n(.*?)\nend", src, flags=re.S).group(1)
    return [(n, t) for n, t in re.findall(r"(\w+)::(\w+)", body)]


@pytest.mark.parametrize("c_name, jl_name", [("pcf_params", "PcfParams"), ("pcf_result", "PcfResult"),
                                             ("pcf_dims", "PcfDims")])
def test_julia_binding_structs_match_the_header(c_name, jl_name):
    """The ccall binding's struct mirrors have the header's fields, in order
    and with matching C types (a missing field would let pcf_params_default
    write past the Julia object)."""
    ctype = {"int": "Cint", "double": "Cdouble"}
    c = [(n, ctype[t]) for n, t in _c_struct_fields(c_name)]
    assert _julia_struct_fields(jl_name) == c


def _header_arity(name):
    src = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    m = re.search(r"\b" + name + r"\s*\(([^;{]*?)\)\s*;", src, flags=re.S)
    assert m, name
    params = m.group(1).strip()
    return 0 if params in ("", "void") else len(params.split(","))


def test_julia_ccalls_bind_declared_symbols_with_their_arity():
    """Every ccall of the Julia binding names a function of the header and
    lists as many argument types as the header has parameters (Julia is not
    installed here, so this is the check that the binding would link)."""
    src = open(JL_CORE).read() + open(JL_EXT).read()
    declared = set(declared_functions())
    calls = re.findall(r"ccall\(\(:(pcf_\w+),\s*LIB\),\s*\w+(?:\{\w+\})?,\s*\((.*?)\),", src, flags=re.S)
    assert len(calls) >= 9
    for name, types in calls:
        assert name in declared, name
        n = len([t for t in re.split(r",\s*", types.strip()) if t])
        assert n == _header_arity(name), (name, n, _header_arity(name))


def test_julia_package_extension_layout():
    """PinCFlowGPU is a Julia package whose extension PinCFlowGPUExt loads with
    PinCFlow (a weak dependency, PinCFlow.jl's own UUID from its Project.toml),
    the mechanism the reference itself uses for CairoMakie (PinCFlowMakieExt).
    The extension adds Float64 methods of the three reference functions and
    falls back to the reference's AbstractFloat methods with `invoke`."""
    import tomllib
    with open(os.path.join(JL_PKG, "Project.toml"), "rb") as fh:
        proj = tomllib.load(fh)
    assert proj["name"] == "PinCFlowGPU"
    assert proj["weakdeps"] == {"PinCFlow": "230a4047-f24c-41d9-8d93-b3b8a5ef3847"}
    assert proj["extensions"] == {"PinCFlowGPUExt": "PinCFlow"}
    core, ext = open(JL_CORE).read(), open(JL_EXT).read()
    assert re.search(r"^module PinCFlowGPU$", core, flags=re.M)
    assert re.search(r"^module PinCFlowGPUExt$", ext, flags=re.M)
    assert not re.search(r"^using PinCFlow\b", core, flags=re.M)  # the core module loads without PinCFlow
    for fn, n in (("PS.solve_poisson!", 4), ("PS.apply_corrector!", 3), ("IN.implicit_integration!", 8)):
        m = re.search(r"^function " + re.escape(fn) + r"\((.*?)\)$", ext, flags=re.M | re.S)
        assert m, fn
        assert len(re.findall(r"::", m.group(1))) == n, fn
        assert "::Float64" in m.group(1)
        assert re.search(r"invoke\(" + re.escape(fn), ext), fn
