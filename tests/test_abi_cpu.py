"""The C ABI library on a machine without a GPU: symbols, struct layout, validation, frame index."""
import ctypes
import re
import shutil
import subprocess
from pathlib import Path

import pytest

from StochasticGSCudaBackend import _abi

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "sgs_b200.h"


def declared_functions() -> list[str]:
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:[a-z_0-9 ]+\*?\s*)\b(sgs_[a-z_0-9]+)\s*\(", text, flags=re.M)))


def test_library_exports_every_declared_function():
    lib = _abi.load()
    names = declared_functions()
    assert len(names) >= 9, names
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) == set(_abi.SIGNATURES), "ctypes declarations out of sync with the header"


def test_struct_layout_matches_the_header(tmp_path):
    """ctypes structures have the sizes and offsets a C compiler gives the header's structs."""
    structs = {
        "sgs_gaussians": _abi.Gaussians, "sgs_camera": _abi.Camera, "sgs_settings": _abi.SettingsC,
        "sgs_history": _abi.HistoryC, "sgs_outputs": _abi.Outputs, "sgs_workspace_layout": _abi.WorkspaceLayout,
        "sgs_conv3x3_args": _abi.Conv3x3Args,
    }
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', 'int main(void) {']
    for cname, cls in structs.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for field, _ in cls._fields_:
            lines.append(f'printf("{cname}.{field} %zu\\n", offsetof({cname}, {field}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    cc = shutil.which("gcc") or "gcc"
    exe = tmp_path / "layout"
    subprocess.run([cc, str(src), "-o", str(exe)], check=True)
    out = dict(line.rsplit(" ", 1) for line in subprocess.run([str(exe)], capture_output=True, text=True,
                                                               check=True).stdout.splitlines())
    for cname, cls in structs.items():
        assert int(out[cname]) == ctypes.sizeof(cls), cname
        for field, _ in cls._fields_:
            assert int(out[f"{cname}.{field}"]) == getattr(cls, field).offset, f"{cname}.{field}"


def _args(n=10, width=64, height=48, ss=1, mode=0, reuse=0, gps=0, hybrid=0):
    fake = 0x10000  # never dereferenced: validation fails or sizes are computed before any launch
    g = _abi.Gaussians(fake, fake, fake, fake, fake, n, 16)
    c = _abi.Camera(fake, fake, width, height, 50.0, 50.0, width / 2, height / 2, 0.2, 100.0)
    s = _abi.SettingsC(0, ss, gps, hybrid, reuse, mode, None, None, 0, 0)
    return g, c, s


def test_workspace_size_and_layout():
    lib = _abi.load()
    g, c, s = _args(n=1000, width=640, height=480)
    size = lib.sgs_workspace_size(ctypes.byref(g), ctypes.byref(c), ctypes.byref(s))
    lay = _abi.WorkspaceLayout()
    assert lib.sgs_get_workspace_layout(ctypes.byref(g), ctypes.byref(c), ctypes.byref(s), ctypes.byref(lay)) == 0
    assert lay.total == size
    n_fb = 640 * 480
    assert lay.samples - lay.framebuffer >= 8 * n_fb
    assert all(v % 256 == 0 for v in (lay.framebuffer, lay.samples, lay.reuse_weights, lay.queue, lay.total))
    g2, c2, s2 = _args(n=1000, width=640, height=480, ss=2, reuse=1)
    size2 = lib.sgs_workspace_size(ctypes.byref(g2), ctypes.byref(c2), ctypes.byref(s2))
    assert size2 >= 4 * 40 * n_fb  # fb + samples + reuse weights at 4x the subpixels


def test_hybrid_gps_queue_holds_the_reference_bin():
    """The hybrid-GPS queue holds min(N, 2^20) entries whatever the framebuffer size, like the
    reference's bin (accumulate_hybrid_gps.cu:22,202): at 1280x720 with supersampling 2 a 1M-Gaussian
    scene bins up to 1M Gaussians. An entry whose chunks would pass 32-bit chunk indices is marked
    unused on the device instead of the queue being shortened."""
    lib = _abi.load()

    def size(n, max_binned=0):
        g, c, s = _args(n=n, width=1280, height=720, ss=2, gps=1, hybrid=1)
        s.max_binned = max_binned
        return lib.sgs_workspace_size(ctypes.byref(g), ctypes.byref(c), ctypes.byref(s))

    entry_bytes = 8 + 16 + 16 + 16 + 4  # key, two geometry float4s, meta, point count
    grown = size(1_000_000) - size(1_000_000, max_binned=500_000)
    assert abs(grown - 500_000 * entry_bytes) <= 5 * 256
    assert size(2_000_000) == size(2_000_000, max_binned=1 << 20)


def test_invalid_arguments_are_rejected_before_any_launch():
    lib = _abi.load()
    h = _abi.HistoryC()
    o = _abi.Outputs(0x10000, 0x10000, 0x10000, 0x10000)

    def call(g, c, s, ws=0x100000, nbytes=1 << 40):
        st = lib.sgs_render(ctypes.byref(g), ctypes.byref(c), ctypes.byref(s), ctypes.byref(h), ctypes.byref(o),
                            ctypes.c_void_p(ws), ctypes.c_size_t(nbytes), None)
        return st, _abi.last_error(lib)

    g, c, s = _args(mode=7)
    st, msg = call(g, c, s)
    assert st == _abi.SGS_ERROR_INVALID_ARGUMENT and "temporal mode" in msg
    g, c, s = _args(width=0)
    assert call(g, c, s)[0] == _abi.SGS_ERROR_INVALID_ARGUMENT
    g, c, s = _args()
    g.sh_bases = 5
    assert "sh_bases" in call(g, c, s)[1]
    g, c, s = _args(mode=1)  # STATIC without a history
    assert call(g, c, s)[0] == _abi.SGS_ERROR_INVALID_ARGUMENT
    g, c, s = _args(reuse=1)  # spatial reuse without k-buffers
    assert call(g, c, s)[0] == _abi.SGS_ERROR_INVALID_ARGUMENT
    g, c, s = _args()
    g.rotations = 0x10004  # misaligned quaternions
    assert "aligned" in call(g, c, s)[1]
    g, c, s = _args()
    assert call(g, c, s, ws=0x100010)[0] == _abi.SGS_ERROR_WORKSPACE  # misaligned workspace
    assert call(g, c, s, nbytes=16)[0] == _abi.SGS_ERROR_WORKSPACE  # too small
    g, c, s = _args(width=1 << 23, height=1 << 12, ss=4)  # framebuffer side beyond exact float range
    assert call(g, c, s)[0] == _abi.SGS_ERROR_INVALID_ARGUMENT


def test_frame_index_and_constants():
    lib = _abi.load()
    assert lib.sgs_k_buffer_size() == 4
    assert lib.sgs_abi_version() == _abi.ABI_VERSION
    lib.sgs_set_frame_index(123)
    assert lib.sgs_get_frame_index() == 123
    lib.sgs_set_frame_index(0xFFFFFFFF)
    assert lib.sgs_get_frame_index() == 0xFFFFFFFF
    lib.sgs_set_frame_index(0)


def test_python_module_mirrors_the_reference_binding():
    import inspect

    import torch

    from StochasticGSCudaBackend import History, Settings, TemporalMode, _C, create_k_buffer, render

    assert _C.k_buffer_size == 4
    assert Settings._fields == ("w2c", "cam_position", "width", "height", "focal_x", "focal_y", "center_x",
                                "center_y", "near_plane", "far_plane", "proper_antialiasing", "supersampling_factor",
                                "use_gps", "hybrid_scheduling", "spatial_reuse")
    assert [m.name for m in TemporalMode] == ["RESET", "STATIC", "REPROJECT"] and int(TemporalMode.REPROJECT) == 2
    assert History._fields == ("image", "depth", "alpha", "weight_mass")
    params = inspect.signature(render).parameters.values()
    positional = [p.name for p in params if p.kind is not inspect.Parameter.KEYWORD_ONLY]
    assert positional == ["means", "scales", "rotations", "opacities", "sh_coefficients", "settings", "k_buffer",
                          "history", "view_to_previous_view", "temporal_mode"]
    # additions are keyword-only with defaults, so every reference call binds unchanged
    extras = [p for p in params if p.kind is inspect.Parameter.KEYWORD_ONLY]
    assert [p.name for p in extras] == ["preactivated", "max_fragments", "max_binned", "quantized"]
    assert [p.default for p in extras] == [None, 0, 0, None]
    assert callable(create_k_buffer)
    with pytest.raises(TypeError):
        _C.render(1, 2, 3)
    cpu = torch.zeros(4, 3)
    with pytest.raises(RuntimeError, match="CUDA"):
        _C.render(cpu, cpu, cpu, cpu, cpu, cpu, cpu, 4, 4, 1.0, 1.0, 2.0, 2.0, 0.1, 10.0, False, 1, False, False,
                  False, torch.empty(0), cpu, cpu, cpu, cpu, cpu, cpu, cpu, 0)


def test_no_alloc_scratch_bounds_hold():
    """The fixed 64 MiB scratch of sgs_render_no_alloc holds what its documentation says: stochastic
    transparency at 1920x1080 for any scene size, hybrid GPS at 1920x1080 up to about 289,000 queue
    entries (max_binned), and not the hybrid-GPS default queue of a 1M-Gaussian scene."""
    lib = _abi.load()
    limit = 64 << 20

    def size(n, gps, hybrid, max_binned=0):
        g, c, s = _args(n=n, width=1920, height=1080, gps=gps, hybrid=hybrid)
        s.max_binned = max_binned
        return lib.sgs_workspace_size(ctypes.byref(g), ctypes.byref(c), ctypes.byref(s))

    for n in (1000, 1 << 18, 6_000_000, 0xFFFFFFFF):
        assert 0 < size(n, 0, 0) <= limit
        assert 0 < size(n, 0, 1) <= limit
    assert size(285_000, 1, 1) <= limit < size(295_000, 1, 1)
    assert size(6_000_000, 1, 1, max_binned=285_000) <= limit
    assert size(1_000_000, 1, 1) > limit


def test_gps_backward_scratch_holds_the_count_law_table():
    """The GPS backward's table of the point count's law (1025 rows x 32 float pairs) sits in the
    fused walk's scratch after the per-pixel sample table: GPS settings add exactly its size."""
    lib = _abi.load()
    table = lib.sgs_gps_count_law_size()
    assert table == 1025 * 32 * 8 and table % 256 == 0
    for ss, n_samples in ((1, 1), (2, 8), (3, 5)):
        _, c, s_st = _args(width=96, height=64, ss=ss)
        _, _, s_gps = _args(width=96, height=64, ss=ss, gps=1)
        _, _, s_hyb = _args(width=96, height=64, ss=ss, gps=1, hybrid=1)
        st = lib.sgs_backward_samples_scratch_size(ctypes.byref(c), ctypes.byref(s_st), n_samples)
        n_fb = 96 * 64 * ss * ss
        align = lambda v: (v + 255) // 256 * 256  # noqa: E731
        assert st == align(8 * n_fb * n_samples) + align(4 * n_fb * n_samples) + align(8 * n_fb)
        assert lib.sgs_backward_samples_scratch_size(ctypes.byref(c), ctypes.byref(s_gps), n_samples) == st + table
        assert lib.sgs_backward_samples_scratch_size(ctypes.byref(c), ctypes.byref(s_hyb), n_samples) == st + table


def test_count_law_and_autograd_reject_bad_input_before_any_launch():
    """sgs_gps_count_law wants an 8-byte aligned buffer; render_samples refuses spatial reuse (its
    samples mix neighbours' winners through the k-buffer) before touching the device."""
    import torch

    from StochasticGSCudaBackend import Settings
    from StochasticGSCudaBackend.autograd import render_samples

    lib = _abi.load()
    assert lib.sgs_gps_count_law(None, None) == _abi.SGS_ERROR_INVALID_ARGUMENT
    assert lib.sgs_gps_count_law(ctypes.c_void_p(0x10004), None) == _abi.SGS_ERROR_INVALID_ARGUMENT
    assert "8-byte aligned" in _abi.last_error(lib)
    params = [torch.zeros((4, 3)), torch.zeros((4, 3)), torch.zeros((4, 4)), torch.zeros((4,)),
              torch.zeros((4, 16, 3))]
    settings = Settings(torch.eye(4), torch.zeros(3), 32, 24, 30.0, 30.0, 16.0, 12.0, 0.2, 100.0, False, 1, False,
                        False, True)
    with pytest.raises(RuntimeError, match="spatial reuse"):
        render_samples(*params, settings, n_samples=2, first_frame=0)
