"""CPU tests of the drop-in boundary: the library loads, exports every entry
point declared in include/*.h, and rejects unsupported problems before any
CUDA call (reference include/conv2d.h:69-70; the reference itself returns 0
for every shape, src/conv2d.cpp:516)."""
import ctypes
import os
import re
import subprocess

import numpy as np

import pytest

from conftest import ROOT


def _declared_functions():
    names = set()
    for h in ("conv2d.h", "winoconv.h"):
        src = open(os.path.join(ROOT, "include", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:int|size_t|void\s*\*?)\s+(\w+)\s*\(", src, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_headers_declare_the_reference_entry_points():
    names = _declared_functions()
    assert "getParamsize" in names and "getkernelInfo" in names
    assert "wino_conv2d_fused" in names


def test_library_exports_every_declared_symbol(wino):
    lib = wino.LIB_PATH
    out = subprocess.run(["nm", "-D", "--defined-only", lib], capture_output=True, text=True,
                         check=True).stdout
    exported = {l.split()[-1] for l in out.splitlines() if l.strip()}
    missing = []
    for name in _declared_functions():
        if name in ("getParamsize", "getkernelInfo"):
            # C++ linkage, as the reference header declares them
            if not any(e.startswith(f"_Z{len(name)}{name}") for e in exported):
                missing.append(name)
        elif name not in exported:
            missing.append(name)
    assert not missing, missing
    # The mangled names a reference caller links against.
    assert "_Z12getParamsizeP9problem_tPi" in exported
    assert "_Z13getkernelInfoP9problem_tP12kernelInfo_tPv" in exported


def test_param_size_is_reference_layout(wino):
    pr = wino.Problem()
    assert wino.get_param_size(pr) == 80  # 6 pointers + 13 shorts on x86-64
    assert ctypes.sizeof(wino.Problem) == 96
    assert ctypes.sizeof(wino.KernelInfo) == 160


def _problem(wino, **kw):
    f = dict(in_=0x1000, weight=0x2000, out=0x3000, transform_pin=0, transform_filter=0x4000,
             mid_result=0, n=2, c=64, h=14, w=14, k=64, r=3, s=3, u=1, v=1, p=1, q=1)
    f.update(kw)
    pr = wino.Problem()
    for k_, v_ in f.items():
        setattr(pr, k_, v_)
    return pr


@pytest.mark.parametrize("field,value,code", [
    ("h", 40000, 2), ("n", 0, 1), ("w", 0, 1), ("r", 0, 1), ("u", 0, 1), ("r", 40, 1),
    ("in_", 0, 1), ("weight", 0, 1), ("out", 0, 1),
])
def test_getkernelinfo_rejects_invalid(wino, field, value, code):
    pr = _problem(wino, **{field: value})
    param = (ctypes.c_char * 80)()
    rc, _ = wino.get_kernel_info(pr, param)
    assert rc == code


@pytest.mark.parametrize("field,value", [
    ("r", 5), ("c", 8), ("c", 3), ("transform_filter", 0),
])
def test_getkernelinfo_sends_other_shapes_to_the_direct_kernel(wino, field, value):
    """Shapes outside the Winograd contract whose implicit-GEMM weights do not
    fit transform_filter (or with no usable transform_filter) get the direct
    kernel in slot 3 and empty kernels elsewhere (needs no GPU: no attribute
    is set)."""
    pr = _problem(wino, **{field: value})
    param = (ctypes.c_char * 80)()
    rc, ki = wino.get_kernel_info(pr, param)
    assert rc == 0
    L = wino.lib()
    L.wino_direct_kernel_ptr.restype = ctypes.c_void_p
    assert ki.slot(3)["kernel"] == L.wino_direct_kernel_ptr()
    assert ki.slot(1)["kernel"] == ki.slot(2)["kernel"] == ki.slot(4)["kernel"]
    dims = np.frombuffer(bytes(param)[48:74], dtype=np.int16)
    n, c, h, w, k, r, s, u, v, p, q, oh, ow = dims
    assert oh == (h - r + 2 * p) // u + 1 and ow == (w - s + 2 * q) // v + 1


def test_igemm_weight_bytes_and_entry_points(wino):
    L = wino.lib()
    # round16(k) rows x r*s*ceil(c/16) K-steps x 32 bytes, then a 128-byte
    # tensor-map slot at a 128-byte boundary
    L.wino_igemm_operand_bytes.restype = ctypes.c_size_t
    L.wino_igemm_map_offset.restype = ctypes.c_size_t
    for (c, k, r, s, ops) in [(64, 128, 3, 3, 128 * 9 * 4 * 32), (24, 40, 3, 3, 48 * 9 * 2 * 32),
                              (3, 64, 7, 7, 64 * 49 * 32), (3, 16, 1, 1, 16 * 1 * 32)]:
        assert L.wino_igemm_operand_bytes(c, k, r, s) == ops
        assert L.wino_igemm_map_offset(c, k, r, s) == (ops + 127) // 128 * 128
        assert L.wino_igemm_weight_bytes(c, k, r, s) == (ops + 127) // 128 * 128 + 128
    d = ctypes.c_void_p(0x10000)
    odd = ctypes.c_void_p(0x10008)
    assert L.wino_igemm_weight_transform(None, d, 16, 16, 3, 3, None) == 1
    assert L.wino_igemm_weight_transform(d, odd, 16, 16, 3, 3, None) == 1   # wprep alignment
    assert L.wino_igemm_weight_transform(d, d, 0, 16, 3, 3, None) == 1
    assert L.wino_conv2d_igemm(None, d, d, 1, 16, 8, 8, 16, 3, 3, 2, 2, 1, 1, None) == 1
    assert L.wino_conv2d_igemm(d, odd, d, 1, 16, 8, 8, 16, 3, 3, 2, 2, 1, 1, None) == 1
    assert L.wino_conv2d_igemm(d, d, d, 1, 16, 8, 8, 16, 9, 9, 1, 1, 0, 0, None) == 1  # filter > input
    # one image of 2^31 input elements: offsets would leave 32 bits
    assert L.wino_conv2d_igemm(d, d, d, 1, 2048, 1024, 1024, 16, 1, 1, 1, 1, 0, 0, None) == 2


def test_igemm_units_and_grid(wino):
    """Units of the persistent implicit GEMM: 128 output pixels (256 when
    K <= 128) x one 256-row block of output channels; the grid is capped at
    the SM count."""
    L = wino.lib()
    L.wino_igemm_units.restype = ctypes.c_longlong
    L.wino_igemm_grid.restype = ctypes.c_uint
    assert L.wino_igemm_units(128, 256, 56, 56) == 128 * 3136 // 128            # K = 256: one block
    assert L.wino_igemm_units(128, 64, 28, 28) == (128 * 784 + 255) // 256      # two pixel halves
    assert L.wino_igemm_units(3, 320, 28, 28) == (3 * 784 + 127) // 128 * 2     # two k-blocks
    assert L.wino_igemm_units(1, 27, 7, 7) == 1                                 # K padded to 32
    assert L.wino_igemm_grid(128, 256, 56, 56, 148) == 148
    assert L.wino_igemm_grid(1, 27, 7, 7, 148) == 1
    assert L.wino_igemm_shape_ok(1, 64, 56, 56, 64, 56, 56) == 1
    assert L.wino_igemm_shape_ok(1, 2048, 1024, 1024, 16, 1024, 1024) == 0      # 2^31 input elements


@pytest.mark.parametrize("x,h,w,r,s,u,v,p,q,flat", [
    (0x1000, 14, 14, 1, 1, 1, 1, 0, 0, 0),     # 1x1 but H*W % 8 != 0: 2-byte gather
    (0x1000, 28, 28, 1, 1, 1, 1, 0, 0, 1),     # 1x1, H*W % 8 == 0: 16-byte pixel octets
    (0x1008, 28, 28, 1, 1, 1, 1, 0, 0, 0),     # misaligned input
    (0x1000, 28, 28, 1, 1, 2, 2, 0, 0, 0),     # stride 2
    (0x1000, 28, 28, 3, 3, 1, 1, 1, 1, 0),     # 3x3
])
def test_igemm_producer_choice(wino, x, h, w, r, s, u, v, p, q, flat):
    """Which pixel-operand producer the implicit GEMM uses: 1 = 16-byte
    pixel octets or TMA boxes (1x1 / stride 1 / pad 0), 0 = 2-byte gathers;
    with K <= 128 (two pixel halves a unit) never TMA."""
    L = wino.lib()
    L.wino_igemm_flat.argtypes = [ctypes.c_void_p] + [ctypes.c_int] * 8
    assert L.wino_igemm_flat(x, h, w, r, s, u, v, p, q) == flat
    L.wino_igemm_mode.argtypes = [ctypes.c_void_p] + [ctypes.c_int] * 9
    assert L.wino_igemm_mode(x, 64, h, w, r, s, u, v, p, q) == flat     # K = 64: octet loads


@pytest.mark.parametrize("field,value", [
    ("s", 1), ("u", 2), ("v", 2), ("p", 0), ("q", 2), ("k", 27), ("c", 24),
])
def test_getkernelinfo_sends_other_shapes_to_the_igemm_kernel(wino, field, value):
    """Shapes outside the Winograd contract whose re-laid-out weights fit
    transform_filter get the weight re-layout in slot 1 and the tensor-core
    implicit GEMM in slot 3 (the CUDA attribute call needs a GPU, so only the
    route is checked here)."""
    pr = _problem(wino, **{field: value})
    assert wino.lib().wino_dropin_route(ctypes.byref(pr)) == 4


def test_check_shape(wino):
    L = wino.lib()
    assert L.wino_check_shape(128, 256, 28, 28, 256) == 0
    assert L.wino_check_shape(1, 48, 7, 7, 48) == 0
    assert L.wino_check_shape(1, 24, 7, 7, 48) == 2
    assert L.wino_ucache_bytes(256, 256, 0) == 16 * 256 * 256 * 2


def test_host_u_cache_layout_is_a_bijection():
    """The tile-major U offset formula visits every element exactly once."""
    import numpy as np
    for K, C in [(32, 16), (48, 32), (16, 48), (144, 32), (272, 16)]:
        seen = np.zeros(16 * K * C, np.int32)
        KB = 128
        for t in range(16):
            for k in range(K):
                for c in range(C):
                    kb, kr = divmod(k, KB)
                    kbs = min(KB, K - kb * KB)
                    cs, cc = divmod(c, 16)
                    off = (kb * KB * 16 * C + (cs * 16 + t) * kbs * 16 + (kr >> 3) * 128 +
                           (cc >> 3) * 64 + (kr & 7) * 8 + (cc & 7))
                    seen[off] += 1
        assert (seen == 1).all()


def test_batch_host_validation(wino):
    """Batch object bookkeeping that needs no GPU: shape checks, the layer
    cap, order permutations, configuration ranges."""
    L = wino.lib()
    h = ctypes.c_void_p(0)
    assert L.wino_batch_create(ctypes.byref(h)) == 0
    dummy = ctypes.c_void_p(0x1000)
    assert L.wino_batch_add_layer(h, dummy, dummy, None, dummy, 2, 64, 14, 14, 64) == 0
    assert L.wino_batch_add_layer(h, dummy, dummy, None, dummy, 2, 24, 14, 14, 64) == 2   # C % 16
    assert L.wino_batch_add_layer(h, None, dummy, None, dummy, 2, 64, 14, 14, 64) == 1    # null input
    assert L.wino_batch_add_layer(h, dummy, dummy, ctypes.c_void_p(0x1008), dummy, 2, 64, 14, 14, 64) == 1
    assert L.wino_batch_add_layer(h, dummy, dummy, None, dummy, 1, 32, 7, 7, 32) == 0
    assert L.wino_batch_num_layers(h) == 2
    bad = (ctypes.c_int * 2)(0, 0)
    good = (ctypes.c_int * 2)(1, 0)
    assert L.wino_batch_set_order(h, bad, 2) == 1
    assert L.wino_batch_set_order(h, good, 2) == 0
    out = (ctypes.c_int * 2)()
    assert L.wino_batch_get_order(h, out, 2) == 0 and list(out) == [1, 0]
    assert L.wino_batch_set_config(h, 0, 4) == 1
    assert L.wino_batch_set_config(h, 2, 0) == 1
    assert L.wino_batch_set_config(h, 1, 3) == 0
    for _ in range(30):
        assert L.wino_batch_add_layer(h, dummy, dummy, None, dummy, 1, 16, 4, 4, 16) == 0
    assert L.wino_batch_add_layer(h, dummy, dummy, None, dummy, 1, 16, 4, 4, 16) == 2     # 33rd
    assert L.wino_batch_destroy(h) == 0


def test_split_configuration_sizes(wino):
    """Host arithmetic of the schedule configurations (no GPU): workspace
    bytes, split counts (every split non-empty) and work blocks."""
    L = wino.lib()
    L.wino_fused_nblocks_cfg.argtypes = [ctypes.c_int] * 6
    L.wino_fused_nblocks_cfg.restype = ctypes.c_longlong
    L.wino_fused_cfg_splits.argtypes = [ctypes.c_int, ctypes.c_int]
    L.wino_fused_nblocks.argtypes = [ctypes.c_int] * 4
    L.wino_fused_nblocks.restype = ctypes.c_longlong
    n, c, h, w, k = 2, 256, 14, 14, 64
    xb = wino.fused_workspace_bytes(n, c, h, w)
    al = lambda b: (b + 255) // 256 * 256
    y32 = n * k * h * w * 4
    assert wino.cfg_workspace_bytes(n, c, h, w, k, 0) == al(xb)
    assert wino.cfg_workspace_bytes(n, c, h, w, k, wino.CFG_KMAJOR) == al(xb)
    assert wino.cfg_workspace_bytes(n, c, h, w, k, wino.CFG_DIRECT) == 0
    assert wino.cfg_workspace_bytes(n, c, h, w, k, wino.cfg_split(1)) == al(xb) + y32
    assert wino.cfg_workspace_bytes(n, c, h, w, k, wino.CFG_DIRECT | wino.cfg_split(2)) == y32
    assert wino.tune_workspace_bytes(n, c, h, w, k) == al(xb) + y32
    # 16 steps: 4^L wanted -> 1, 4, 16, 16 splits; 1 step: never split
    assert [L.wino_fused_cfg_splits(256, wino.cfg_split(l)) for l in range(4)] == [1, 4, 16, 16]
    assert [L.wino_fused_cfg_splits(16, wino.cfg_split(l)) for l in range(4)] == [1, 1, 1, 1]
    assert L.wino_fused_cfg_splits(48, wino.cfg_split(1)) == 3          # 3 steps, one each
    assert wino.cfg_workspace_bytes(1, 16, 8, 8, 16, wino.cfg_split(3)) == al(wino.fused_workspace_bytes(1, 16, 8, 8))
    base = L.wino_fused_nblocks(n, h, w, k)
    assert L.wino_fused_nblocks_cfg(n, c, h, w, k, wino.cfg_split(2)) == 16 * base
    assert L.wino_fused_nblocks_cfg(n, c, h, w, k, wino.CFG_KMAJOR) == base
    assert wino.cfg_workspace_bytes(n, 24, h, w, k, 0) == 0               # bad shape


def test_ucache_load_refuses_missing_and_foreign_files(wino, tmp_path):
    """No GPU needed: the header is checked before any device copy."""
    L = wino.lib()
    dummy = ctypes.c_void_p(0x1000)
    missing = os.fsencode(str(tmp_path / "none.bin"))
    assert L.wino_ucache_load(missing, dummy, 32, 32, 1) == 7           # WINO_EIO
    p = tmp_path / "foreign.bin"
    p.write_bytes(b"NOTAUCAC" + bytes(40))
    assert L.wino_ucache_load(os.fsencode(str(p)), dummy, 32, 32, 1) == 6  # WINO_ESTALE
    assert L.wino_ucache_load(os.fsencode(str(p)), dummy, 32, 24, 1) == 2  # bad shape
    assert L.wino_ucache_load(None, dummy, 32, 32, 1) == 1


def test_new_entry_points_validate_before_launching(wino):
    """Argument checks of the extension entry points return codes without any
    CUDA call (so they run here without a GPU)."""
    L = wino.lib()
    d = ctypes.c_void_p(0x10000)
    odd = ctypes.c_void_p(0x10002)
    # fused epilogue: null pointers, misaligned workspace/residual, bad shape
    assert L.wino_conv2d_fused_epilogue(None, d, d, d, None, None, 0, 1, 16, 8, 8, 16, None) == 1
    assert L.wino_conv2d_fused_epilogue(d, d, odd, d, None, None, 0, 1, 16, 8, 8, 16, None) == 1
    assert L.wino_conv2d_fused_epilogue(d, d, d, d, None, odd, 0, 1, 16, 8, 8, 16, None) == 1
    assert L.wino_conv2d_fused_epilogue(d, d, d, d, None, None, 0, 1, 24, 8, 8, 16, None) == 2
    # direct conv: general shapes accepted by validation, invalid ones refused
    assert L.wino_conv2d_direct(None, d, d, 1, 3, 8, 8, 4, 3, 3, 1, 1, 1, 1, None) == 1
    assert L.wino_conv2d_direct(d, d, d, 1, 3, 2, 2, 4, 5, 5, 1, 1, 0, 0, None) == 1   # filter > input
    assert L.wino_conv2d_direct(d, d, d, 1, 3, 8, 8, 4, 3, 3, 0, 1, 1, 1, None) == 1   # stride 0
    assert L.wino_conv2d_direct(d, d, d, 1, 3, 40000, 8, 4, 3, 3, 1, 1, 1, 1, None) == 2
    # variants: fp8 needs C % 32 == 0; bad variant id
    assert L.wino_variant_workspace_bytes(2, 1, 48, 8, 8, 16) == 0
    assert L.wino_variant_workspace_bytes(9, 1, 64, 8, 8, 16) == 0
    assert L.wino_conv2d_variant(9, d, d, d, d, 1, 64, 8, 8, 16, None) == 1
    assert L.wino_conv2d_variant(0, d, d, d, odd, 1, 64, 8, 8, 16, None) == 1           # ws alignment
    # schedule configurations: cfg out of range, missing workspace
    assert L.wino_conv2d_fused_cfg(d, d, None, d, 1, 64, 8, 8, 16, 16, None) == 1
    assert L.wino_conv2d_fused_cfg(d, d, None, d, 1, 64, 8, 8, 16, 0, None) == 1
    assert L.wino_conv2d_fused_ws(d, d, None, d, 1, 64, 8, 8, 16, None) == 1


def test_f4_entry_points_validate_and_size(wino):
    """Winograd F(4x4,3x3) entry points: workspace arithmetic and the argument
    checks that return before any CUDA call."""
    L = wino.lib()
    d = ctypes.c_void_p(0x10000)
    odd = ctypes.c_void_p(0x10010)          # 16- but not 256-byte aligned
    r256 = lambda b: (b + 255) // 256 * 256
    # N128 C256 H28 K256: 7 x 7 tiles per image -> 6272 tiles, 49 blocks of 128
    ntp = 49 * 128
    for hilo, cr in ((0, 256), (1, 768)):
        u, v, m = r256(36 * 256 * cr * 2), r256(36 * ntp * cr * 2), r256(36 * 256 * ntp * 4)
        assert L.wino_f4_filter_bytes(256, 256, hilo) == u
        assert L.wino_f4_workspace_bytes(128, 256, 28, 28, 256, hilo) == u + v + m
    full = L.wino_f4_workspace_bytes(1, 16, 8, 8, 16, 1)
    fb = L.wino_f4_filter_bytes(16, 16, 1)
    assert L.wino_f4_filter_transform(None, 16, 16, 1, d, fb, None) == 1
    assert L.wino_f4_filter_transform(d, 16, 24, 1, d, fb, None) == 2        # C % 16
    assert L.wino_f4_filter_transform(d, 16, 16, 2, d, fb, None) == 1        # hilo not 0/1
    assert L.wino_f4_filter_transform(d, 16, 16, 1, d, fb - 1, None) == 5    # workspace too small
    assert L.wino_f4_filter_transform(d, 16, 16, 1, odd, fb, None) == 1      # alignment
    assert L.wino_conv2d_f4(None, d, 1, 16, 8, 8, 16, 1, d, full, None) == 1
    assert L.wino_conv2d_f4(d, d, 1, 16, 8, 8, 24, 1, d, full, None) == 2    # K % 16
    assert L.wino_conv2d_f4(d, d, 0, 16, 8, 8, 16, 1, d, full, None) == 1    # n = 0
    assert L.wino_conv2d_f4(d, d, 1, 16, 8, 8, 16, 1, d, full - 1, None) == 5
    assert L.wino_conv2d_f4(d, d, 1, 16, 8, 8, 16, 1, odd, full, None) == 1


def _xr_bytes(n, c, h, w):
    """Row-transformed pre-pass records of the tap-pair route: per image and
    16-channel block 4*ceil(h/2) rows of 64*(ceil(w/2) + 1) bytes."""
    return n * (c // 16) * 4 * ((h + 1) // 2) * 64 * ((w + 1) // 2 + 1)


def _pre_bytes(L, n, c, h, w):
    """Pre-pass output of the kernel the build routes C to: transformed tiles
    V2 for the bulk-copy-fed resident-U kernel, row-transformed records for
    the producer-fed resident-U and tap-pair kernels, channel-blocked records
    for the streamed-U kernel."""
    kp = L.wino_twostage_gemm_kernel_ptr_for(c)
    if kp == L.wino_twostage_resv_kernel_ptr():
        tiles8 = (n * ((h + 1) // 2) * ((w + 1) // 2) + 7) // 8 * 8
        return 16 * tiles8 * c * 2
    if kp in (L.wino_twostage_pair_kernel_ptr(), L.wino_twostage_res_kernel_ptr()):
        return _xr_bytes(n, c, h, w)
    return L.wino_xb_bytes(n, c, h, w)


def test_twostage_entry_points_validate_and_size(wino):
    """Two-stage path: workspace = pre-pass records (row-transformed for the
    resident-U and tap-pair kernels, channel-blocked for the streamed-U
    kernel; 256-byte aligned) + 16*K*tiles fp16 of M; argument checks return
    before any CUDA call."""
    L = wino.lib()
    d = ctypes.c_void_p(0x10000)
    odd = ctypes.c_void_p(0x10010)
    r256 = lambda b: (b + 255) // 256 * 256
    # N128 C256 H28 K256: 25088 tiles; M = 16*256*25088*2 bytes = the reference's mid_result
    m = 16 * 256 * 25088 * 2
    assert m == 4 * 256 * 28 * 28 * 128 * 2
    assert L.wino_twostage_workspace_bytes(128, 256, 28, 28, 256) == r256(_pre_bytes(L, 128, 256, 28, 28)) + m
    # every kind of pre-pass output fits the reference harness's transform_pin (4*h*h*n*c fp16)
    assert 16 * 25088 * 256 * 2 == 4 * 28 * 28 * 128 * 256 * 2
    assert _xr_bytes(128, 256, 28, 28) <= 4 * 28 * 28 * 128 * 256 * 2
    assert L.wino_xb_bytes(128, 256, 28, 28) <= 4 * 28 * 28 * 128 * 256 * 2
    # odd sizes: tiles = n * ceil(h/2) * ceil(w/2)
    assert (L.wino_twostage_workspace_bytes(3, 48, 9, 7, 144)
            == r256(_pre_bytes(L, 3, 48, 9, 7)) + 16 * 144 * (3 * 5 * 4) * 2)
    # C > 256: always the streamed-U kernel on the channel-blocked records
    assert L.wino_twostage_gemm_kernel_ptr_for(272) == L.wino_twostage_stream_kernel_ptr()
    assert (L.wino_twostage_workspace_bytes(2, 272, 6, 8, 48)
            == r256(L.wino_xb_bytes(2, 272, 6, 8)) + 16 * 48 * (2 * 3 * 4) * 2)
    assert L.wino_twostage_workspace_bytes(1, 24, 8, 8, 16) == 0          # C % 16
    assert L.wino_conv2d_twostage(None, d, d, d, 1, 16, 8, 8, 16, None) == 1
    assert L.wino_conv2d_twostage(d, d, odd, d, 1, 16, 8, 8, 16, None) == 1  # workspace alignment
    assert L.wino_conv2d_twostage(d, d, d, d, 1, 16, 8, 8, 24, None) == 2    # K % 16
    assert L.wino_twostage_stage(3, d, d, d, d, 1, 16, 8, 8, 16, None) == 1  # no such stage
    assert L.wino_twostage_stage(-1, d, d, d, d, 1, 16, 8, 8, 16, None) == 1
    # one 16384 x 16384 image: its blocked-input record block exceeds 2^31 bytes
    assert L.wino_twostage_workspace_bytes(1, 16, 16384, 16384, 16) == 0
    assert L.wino_conv2d_twostage(d, d, d, d, 1, 16, 16384, 16384, 16, None) == 2


@pytest.mark.parametrize("kw,route", [
    (dict(h=12, w=10, transform_pin=0x100000, mid_result=0x200000), 3),   # even H, W: two-stage
    (dict(h=12, w=9, transform_pin=0x100000, mid_result=0x200000), 2),    # odd W: M would not fit
    (dict(h=11, w=10, transform_pin=0x100000, mid_result=0x200000), 2),   # odd H
    (dict(h=12, w=10, transform_pin=0x100000, mid_result=0), 2),          # no mid_result
    (dict(h=12, w=10, transform_pin=0, mid_result=0x200000), 1),          # no transform_pin
    (dict(h=12, w=10, transform_pin=0x100008, mid_result=0x200000), 1),   # misaligned transform_pin
    (dict(h=12, w=10, transform_pin=0x100000, mid_result=0x200000, transform_filter=0), 0),
    (dict(h=12, w=10, transform_pin=0x100000, mid_result=0x200000, r=5, s=5, p=2, q=2), 0),
    (dict(h=12, w=10, transform_pin=0x100000, mid_result=0x200000, c=24), 4),
    (dict(h=12, w=10, transform_pin=0x100000, mid_result=0x200000, u=2, v=2), 4),
    (dict(h=12, w=10, r=1, s=1, p=0, q=0), 4),                           # 1x1
    (dict(h=12, w=10, r=1, s=1, p=0, q=0, transform_filter=0x4008), 0),  # misaligned transform_filter
    (dict(h=12, w=10, c=3, r=7, s=7, p=3, q=3, u=2, v=2), 0),            # weights do not fit
])
def test_dropin_route_selection(wino, kw, route):
    """Which kernels getkernelInfo will put in the slots (decided without CUDA
    calls): 0 direct, 1 fused on the NCHW input, 2 fused after the pre-pass,
    3 two-stage (M in the caller's mid_result), 4 tensor-core implicit GEMM."""
    pr = _problem(wino, **{"n": 2, "c": 32, "k": 32, **kw})
    assert wino.lib().wino_dropin_route(ctypes.byref(pr)) == route


def test_dropin_route_rejects_invalid(wino):
    pr = _problem(wino, n=0)
    assert wino.lib().wino_dropin_route(ctypes.byref(pr)) == -1
    assert wino.lib().wino_dropin_route(None) == -1


def test_twostage_f8_entry_points_validate_and_size(wino):
    """fp8 two-stage path: C a multiple of 32 up to 256, K a multiple of 16;
    workspace = channel maxima + su + U terms + V2 terms + M (each 256-byte
    aligned); argument checks return before any CUDA call."""
    L = wino.lib()
    d = ctypes.c_void_p(0x10000)
    odd = ctypes.c_void_p(0x10010)
    r256 = lambda b: (b + 255) // 256 * 256
    assert L.wino_twostage_f8_workspace_bytes(2, 48, 8, 8, 32, 1) == 0     # C % 32
    assert L.wino_twostage_f8_workspace_bytes(2, 288, 8, 8, 32, 1) == 0    # C > 256
    assert L.wino_twostage_f8_workspace_bytes(2, 64, 8, 8, 24, 1) == 0     # K % 16
    assert L.wino_twostage_f8_workspace_bytes(2, 64, 8, 8, 32, 2) == 0     # hilo 0 or 1
    tiles8 = (2 * 4 * 4 + 7) // 8 * 8
    for hilo, terms in ((1, 2), (0, 1)):
        assert (L.wino_twostage_f8_workspace_bytes(2, 64, 8, 8, 32, hilo)
                == r256(64 * 4) + r256(16 * 32 * 4) + r256(16 * 32 * 64 * terms) + r256(16 * tiles8 * 64 * terms)
                + 16 * 32 * 32 * 2)
    assert L.wino_conv2d_twostage_f8(None, d, d, d, 2, 64, 8, 8, 32, 1, None) == 1
    assert L.wino_conv2d_twostage_f8(d, d, odd, d, 2, 64, 8, 8, 32, 1, None) == 1   # workspace alignment
    assert L.wino_conv2d_twostage_f8(d, d, d, d, 2, 48, 8, 8, 32, 1, None) == 2     # C % 32
