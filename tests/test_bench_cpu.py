"""Host-side pieces of bench.py that need no GPU: the L2 read probe compiles
for sm_100a, the measured-traffic tables cover every stage the roofline can
name, and the wavefront traces' algorithmic bytes match their queue I/O."""
from __future__ import annotations

import pytest

import bench


def test_l2_probe_compiles_for_sm100a():
    nvrtc = pytest.importorskip("cuda.bindings.nvrtc")
    err, prog = nvrtc.nvrtcCreateProgram(bench.L2_PROBE_SRC, b"l2_probe.cu", 0, [], [])
    assert err == nvrtc.nvrtcResult.NVRTC_SUCCESS
    opts = [b"--gpu-architecture=sm_100a"]
    assert nvrtc.nvrtcCompileProgram(prog, len(opts), opts)[0] == nvrtc.nvrtcResult.NVRTC_SUCCESS
    err, size = nvrtc.nvrtcGetCUBINSize(prog)
    assert err == nvrtc.nvrtcResult.NVRTC_SUCCESS and size > 0


def test_traffic_tables_cover_the_stages():
    # the render roofline picks its dominant stage among these names
    assert set(bench.RENDER_DRAM_BYTES_PER_UNIT) == {
        "k_logic", "k_shade (all kinds)", "k_trace<closest> (extension queue)", "k_trace<any> (shadow queue)"}
    # and the inverse roofline among these
    assert set(bench.ADJ_DRAM_BYTES_PER_UNIT) == {
        "k_logic (adjoint)", "k_shade (adjoint)", "k_trace closest (extension)", "k_trace any (shadow)"}
    for table in (bench.RENDER_DRAM_BYTES_PER_UNIT, bench.ADJ_DRAM_BYTES_PER_UNIT):
        assert all(v > 0 for v in table.values())
    assert bench.CACHE_INFER_DRAM_BYTES_PER_QUERY > 0


def test_wavefront_trace_bytes():
    # tagged queue entry: 32 B ray + 4 B tag in; 16 B hit or 1 B answer out
    assert bench.WF_CLOSEST_BYTES == 52 and bench.WF_ANY_BYTES == 37
    assert bench.RAY_BYTES + bench.HIT_BYTES == 48


def test_checkpoints_grow_by_about_a_quarter():
    c = bench.checkpoints(1024)
    assert c[0] == 1 and c[-1] <= 1024
    assert all(b > a for a, b in zip(c, c[1:]))
    assert all(b <= max(a + 1, round(a * 1.25)) for a, b in zip(c, c[1:]))
