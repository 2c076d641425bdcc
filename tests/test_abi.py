"""The C-ABI library builds, loads and exports every entry point that
include/pfoam.h declares (no compute calls: this runs without a GPU)."""

import ctypes
import os
import re

from tests.conftest import ROOT


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "pfoam.h")).read()
    return sorted(set(re.findall(r"^PF_API\s+[\w\s\*]+?\b(pf_\w+)\s*\(", src, flags=re.M)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "pf_raster_forward" in syms and "pf_raster_backward" in syms and "pf_bin" in syms
    assert len(syms) >= 15


def test_library_exports_every_declared_symbol():
    from powerfoam_b200 import _lib

    lib = _lib.load()
    for s in declared_symbols():
        assert hasattr(lib, s), s
    assert lib.pf_abi_version() == 4
    # every binding in the Python layer names a declared symbol
    assert set(_lib.exported_symbols()) <= set(declared_symbols())


def test_argument_errors_are_reported_without_a_gpu():
    from powerfoam_b200 import _lib

    lib = _lib.load()
    n = ctypes.c_size_t(0)
    assert lib.pf_bin_workspace_size(-1, 0, 0, ctypes.byref(n)) == _lib.PF_ERR_ARGS
    assert b"bad arguments" in lib.pf_last_error()
    assert lib.pf_bin_workspace_size(1000, 5000, 100, ctypes.byref(n)) == 0 and n.value > 0
    assert lib.pf_raster_forward(None, 0, *([None] * 11)) == _lib.PF_ERR_ARGS


def test_oracle_library_loads():
    from oracle import oracle as orc

    lib = orc.lib()
    for s in ["orc_bin_f32", "orc_raster_forward_f32", "orc_raster_backward_f64", "orc_trace_forward_f32"]:
        assert hasattr(lib, s)


def test_trace_backward_workspace_size_without_a_gpu():
    """The tracer adjoint's workspace: 48-byte records per pixel slot (8 x 8
    tiles) and segment slot plus counts, overflow list and states; segment
    counts outside [0, 65535] are rejected."""
    from powerfoam_b200 import _lib

    lib = _lib.load()
    inp = _lib.PfTraceInputs()
    inp.cam.width, inp.cam.height = 30, 17  # 4 x 3 tiles: 768 slots
    n = ctypes.c_size_t(0)
    _lib.call("pf_trace_backward_workspace_size", ctypes.byref(inp), 0, ctypes.byref(n))
    base = n.value
    assert base >= 768 * (4 + 4 + 48)
    _lib.call("pf_trace_backward_workspace_size", ctypes.byref(inp), 10, ctypes.byref(n))
    assert n.value - base >= 768 * 10 * 48 and n.value % 256 == 0
    for kb in (-1, 65536):
        assert lib.pf_trace_backward_workspace_size(ctypes.byref(inp), kb, ctypes.byref(n)) == _lib.PF_ERR_ARGS
    inp.cam.width = 0
    assert lib.pf_trace_backward_workspace_size(ctypes.byref(inp), 4, ctypes.byref(n)) == _lib.PF_ERR_ARGS


def test_struct_layouts_match_the_header(tmp_path):
    """Every ctypes mirror in the Python layer has the C struct's size and
    field offsets (a C program compiled against include/pfoam.h prints them)."""
    import shutil
    import subprocess

    import pytest

    from powerfoam_b200 import _lib

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    mirrors = {"pf_camera": _lib.PfCamera, "pf_raster_inputs": _lib.PfRasterInputs,
               "pf_trace_inputs": _lib.PfTraceInputs, "pf_batch_scene": _lib.PfBatchScene,
               "pf_batch_view": _lib.PfBatchView, "pf_batch_schedule": _lib.PfBatchSchedule}
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "pfoam.h"', "int main(void) {"]
    for cname, py in mirrors.items():
        lines.append(f'    printf("{cname} sizeof %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'    printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["    return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run([cc, "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l.strip()}
    for cname, py in mirrors.items():
        assert got[(cname, "sizeof")] == ctypes.sizeof(py), cname
        for fname, _ in py._fields_:
            assert got[(cname, fname)] == getattr(py, fname).offset, (cname, fname)


def test_batch_argument_checks_without_a_gpu():
    """pf_batch_render checks its scene and views before any CUDA call:
    record groups must start at 0 and grow by at most one per view, the
    segment buffer must be 16-byte aligned and its capacity below 2^31.
    (The pointers below are placeholders: nothing dereferences them.)"""
    from powerfoam_b200 import _lib

    lib = _lib.load()
    fake = 1 << 20  # a 16-byte-aligned placeholder address

    def make(groups, segments=fake, capacity=1024):
        sc = _lib.PfBatchScene()
        sc.n_sites, sc.n_prims = 8, 16
        for f in ("spheres", "nsigmas", "texel_sites", "texel_height", "adjacency", "adjacency_offsets",
                  "adjacency_diff", "segment_masks", "segment_offsets", "segment_count"):
            setattr(sc, f, fake)
        sc.segments, sc.segment_capacity, sc.segment_planes = segments, capacity, 1
        views = (_lib.PfBatchView * len(groups))()
        for v, g in enumerate(groups):
            w = views[v]
            w.cam.width, w.cam.height = 24, 16
            for f in ("tile_offsets", "tile_prims", "texel_rgb", "target", "color", "log_t", "normal_distance",
                      "normal", "grad_color", "contrib", "early_stop", "tile_contrib_pairs", "grad_texel_rgb"):
                setattr(w, f, fake)
            w.segment_pair_base, w.segment_pairs, w.segment_group = 64 * v, 64, g
        return sc, views

    def render(sc, views):
        return lib.pf_batch_render(ctypes.byref(sc), views, len(views), 8, 1, 0, 0, None, 0, None, None, None, None,
                                   None, None, None, None, None)

    for groups in ([0, 2, 2], [1, 1, 1], [0, 1, 0]):
        assert render(*make(groups)) == _lib.PF_ERR_ARGS
        assert b"segment groups" in lib.pf_last_error()
    assert render(*make([0, 0, 1], segments=fake + 4)) == _lib.PF_ERR_ARGS
    assert b"16-byte alignment" in lib.pf_last_error()
    assert render(*make([0, 0, 1], capacity=1 << 31)) == _lib.PF_ERR_ARGS
    # well-formed views pass the checks and stop at the missing workspace and outputs
    assert render(*make([0, 1, 1])) == _lib.PF_ERR_ARGS
    assert b"missing argument" in lib.pf_last_error()


def test_raster_segment_argument_checks_without_a_gpu():
    """pf_raster_forward refuses segment records without masks, offsets or a
    counter, off 16-byte alignment, with a capacity of 2^31 or more, or at
    tile width 32, before any CUDA call (placeholder pointers, never
    dereferenced)."""
    from powerfoam_b200 import _lib

    lib = _lib.load()
    fake = 1 << 20

    def inputs(**over):
        inp = _lib.PfRasterInputs()
        inp.cam.width, inp.cam.height = 24, 16
        inp.tile_width, inp.n_sites, inp.n_prims = 8, 8, 16
        for f in ("spheres", "nsigmas", "texel_sites", "texel_rgb", "texel_height", "adjacency",
                  "adjacency_offsets", "adjacency_diff", "tile_offsets", "tile_prims", "segments", "segment_masks",
                  "segment_offsets", "segment_count"):
            setattr(inp, f, fake)
        inp.segment_pairs, inp.segment_capacity, inp.segment_planes = 64, 1024, 1
        for k, v in over.items():
            setattr(inp, k, v)
        return inp

    for over in (dict(segment_masks=None), dict(segment_count=None), dict(segments=fake + 8),
                 dict(segment_capacity=1 << 31), dict(segment_capacity=-1), dict(tile_width=32)):
        inp = inputs(**over)
        assert lib.pf_raster_forward(ctypes.byref(inp), 0, *([None] * 11)) == _lib.PF_ERR_ARGS, over
        assert b"segment" in lib.pf_last_error(), over
