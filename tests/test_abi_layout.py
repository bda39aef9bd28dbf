"""Struct layout of the C-ABI against its bindings (CPU only).

A small C program compiled against include/tpagmg.h prints sizeof and
offsetof of every field of the structs that cross the boundary.  The ctypes
mirror (tpagmg._lib, tpagmg.projection) and the Julia stub in INTEGRATION.md
must declare the same fields in the same order at the same offsets: a missing
trailing field makes the library write past the caller's struct, a missing
middle field shifts every later one."""
import pathlib
import re
import subprocess

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]

STRUCTS = {
    "tpa_stats": ["cycles", "converged", "compatible", "restarts", "initial_l2", "initial_linf", "final_l2",
                  "final_linf", "target_linf", "residual_scale", "removed_rhs_mean", "device_ms",
                  "kernel_launches", "precision", "removed_rhs_max_component_mean"],
    "tpa_multigrid_options": ["coarse_size", "pre_sweeps", "post_sweeps", "max_levels", "smoother"],
    "tpa_tune_config": ["tail_cells", "tail_ctas", "structured", "vectorized", "pdl", "fuse_restrict",
                        "persistent", "tiles", "ms_per_vcycle"],
    "tpa_projection_options": ["dt", "tolerance", "reference_dt", "inherited_divergence", "max_cycles",
                               "compatibility", "precision", "prepared"],
    "tpa_cmdgfm_system": ["np", "nx", "row_ptr", "col", "val", "rhs", "pressure_cell", "pressure_anchor",
                          "defect_weight", "na", "extra_row_ptr", "extra_col", "extra_val", "extra_rhs",
                          "extra_weight", "row_scale", "col_scale", "drop_tolerance", "tolerance",
                          "max_iterations", "precision", "initial_pressure", "warm_start"],
    "tpa_cmdgfm_stats": ["converged", "iterations", "attempts", "kernel_launches", "initial_residual",
                         "final_residual", "pressure_defect", "jump_defect", "anchor_defect", "setup_ms",
                         "device_ms", "factor_entries", "lower_levels", "upper_levels", "inverse_entries",
                         "initial_guess_used"],
}


@pytest.fixture(scope="module")
def c_layout(tmp_path_factory):
    d = tmp_path_factory.mktemp("abi")
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "tpagmg.h"', "int main(void) {"]
    for s, fields in STRUCTS.items():
        lines.append(f'    printf("{s} size %zu\\n", sizeof({s}));')
        for f in fields:
            lines.append(f'    printf("{s} {f} %zu\\n", offsetof({s}, {f}));')
    lines += ["    return 0;", "}"]
    src = d / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = d / "layout"
    subprocess.check_call(["gcc", "-std=c11", "-Wall", "-Werror", "-I", str(ROOT / "include"), str(src), "-o", str(exe)])
    out = {}
    for line in subprocess.check_output([str(exe)], text=True).splitlines():
        s, f, v = line.split()
        out[(s, f)] = int(v)
    return out


def test_header_declares_the_listed_fields(c_layout):
    for s, fields in STRUCTS.items():
        assert [f for (t, f) in c_layout if t == s and f != "size"] == fields


def test_ctypes_structs_match_header(c_layout):
    from tpagmg import _lib
    from tpagmg.projection import ProjectionOptions
    for s, cls in (("tpa_stats", _lib.StatsC), ("tpa_multigrid_options", _lib.MultigridOptionsC),
                   ("tpa_tune_config", _lib.TuneC), ("tpa_projection_options", ProjectionOptions),
                   ("tpa_cmdgfm_system", _lib.CmdgfmSystemC), ("tpa_cmdgfm_stats", _lib.CmdgfmStatsC)):
        import ctypes
        assert ctypes.sizeof(cls) == c_layout[(s, "size")], s
        assert [f[0] for f in cls._fields_] == STRUCTS[s], s
        for f in STRUCTS[s]:
            assert getattr(cls, f).offset == c_layout[(s, f)], (s, f)


JULIA_SIZES = {"Int32": 4, "Float64": 8, "Ptr{Float64}": 8, "Ptr{Cvoid}": 8, "Int64": 8, "Ptr{Int64}": 8,
               "Ptr{Int32}": 8}


def _julia_structs():
    text = (ROOT / "INTEGRATION.md").read_text()
    out = {}
    for name, body in re.findall(r"^struct (\w+)\n(.*?)^end", text, re.S | re.M):
        fields = []
        for stmt in re.sub(r"#.*", "", body).replace("\n", ";").split(";"):
            stmt = stmt.strip()
            if stmt:
                f, t = stmt.split("::")
                fields.append((f.strip(), t.strip()))
        out[name] = fields
    return out


def test_julia_stub_matches_header(c_layout):
    """The Julia stub's isbits structs (C layout: each field aligned to its
    size, the struct to its largest field) equal the header's."""
    julia = _julia_structs()
    for jname, cname in (("TpaStats", "tpa_stats"), ("TpaMultigridOptions", "tpa_multigrid_options"),
                         ("TpaProjectionOptions", "tpa_projection_options"),
                         ("TpaCmdgfmSystem", "tpa_cmdgfm_system"), ("TpaCmdgfmStats", "tpa_cmdgfm_stats")):
        fields = julia[jname]
        assert [f for f, _ in fields] == STRUCTS[cname], jname
        off, align = 0, 1
        for f, t in fields:
            size = JULIA_SIZES[t]
            off = (off + size - 1) // size * size
            assert off == c_layout[(cname, f)], (jname, f)
            off += size
            align = max(align, size)
        assert (off + align - 1) // align * align == c_layout[(cname, "size")], jname


def test_julia_stub_passes_options_as_struct():
    """tpa_build_hierarchy takes a tpa_multigrid_options*: the stub passes a
    Ref of the five-field struct, not a bare Int32 vector."""
    text = (ROOT / "INTEGRATION.md").read_text()
    call = text[text.index("(:tpa_build_hierarchy"):]
    call = call[:call.index("\n")]
    assert "Ref{TpaMultigridOptions}" in call
