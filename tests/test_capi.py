"""The C ABI without a GPU: every declared entry point is exported and bound,
and the host-side logic (defaults, the STANDALONE block enumeration, the
decision over results) equals the oracle's."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

import oracle
import rivet_h26x_codecs_b200.capi as capi
import rivet_h26x_codecs_b200.host as host

HEADER = Path(__file__).resolve().parents[1] / "include" / "rivet_me.h"


def declared():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return sorted(set(re.findall(r"\b(rme_[a-z0-9_]+)\s*\(", text)))


def test_the_library_exports_every_declared_entry_point():
    names = declared()
    assert len(names) >= 25
    lib = capi.lib()
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(capi.SIGNATURES), set(names) ^ set(capi.SIGNATURES)


def test_the_rust_declarations_match_the_header():
    """The Rust FFI module (include/rivet_me_sys.rs) declares every entry
    point with the header's parameter count, and the ctypes binding agrees
    on it too."""
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    c_args = {n: (0 if a.strip() in ("", "void") else a.count(",") + 1)
              for n, a in re.findall(r"\b(rme_[a-z0-9_]+)\s*\(([^;]*?)\)\s*;", text)}
    sys_rs = (HEADER.parent / "rivet_me_sys.rs").read_text()
    rust = {n: len(re.findall(r"\b\w+\s*:", a)) for n, a in re.findall(r"pub fn (rme_[a-z0-9_]+)\(([^)]*)\)", sys_rs)}
    assert set(c_args) == set(declared())
    assert {n: c_args[n] for n in rust} == rust and set(rust) == set(c_args), set(c_args) ^ set(rust)
    assert {n: len(capi.SIGNATURES[n][1]) for n in c_args} == c_args
    # and every struct, field for field in the header's order
    rs_structs = {n: re.findall(r"pub (?:r#)?(\w+)\s*:", body)
                  for n, body in re.findall(r"pub struct (rme_[a-z0-9_]+)\s*\{(.*?)\}", sys_rs, flags=re.S)}
    assert set(rs_structs) == set(_STRUCTS), set(rs_structs) ^ set(_STRUCTS)
    for cname, pyname in _STRUCTS.items():
        assert rs_structs[cname] == [f for f, _ in getattr(capi, pyname)._fields_], cname


_STRUCTS = {"rme_mv": "Mv", "rme_picture_desc": "PictureDesc", "rme_params": "Params", "rme_job": "Job",
            "rme_result": "Result", "rme_frame": "Frame", "rme_stats": "Stats", "rme_bi_job": "BiJob",
            "rme_h264_bi_job": "H264BiJob", "rme_serve_opts": "ServeOpts", "rme_completion": "Completion",
            "rme_plane_set": "PlaneSet"}


def test_every_struct_matches_the_c_compiler(tmp_path):
    """Each struct of the header, compiled by the C compiler, has the size
    and the field offsets of its ctypes mirror."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    assert set(re.findall(r"\}\s*(rme_[a-z0-9_]+)\s*;", text)) == set(_STRUCTS)
    lines = ["#include <stdio.h>", "#include <stddef.h>", f'#include "{HEADER}"', "int main(void) {"]
    for cname, pyname in _STRUCTS.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for field, _ in getattr(capi, pyname)._fields_:
            lines.append(f'  printf("{cname} {field} %zu\\n", offsetof({cname}, {field}));')
    lines += ["  return 0;", "}"]
    (tmp_path / "layout.c").write_text("\n".join(lines) + "\n")
    subprocess.run([cc, "-std=c11", "-o", str(tmp_path / "layout"), str(tmp_path / "layout.c")], check=True)
    out = subprocess.run([str(tmp_path / "layout")], check=True, capture_output=True, text=True).stdout
    for line in out.splitlines():
        cname, what, val = line.split()
        cls = getattr(capi, _STRUCTS[cname])
        got = C.sizeof(cls) if what == "size" else getattr(cls, what).offset
        assert got == int(val), f"{cname}.{what}: ctypes {got}, C {val}"


def test_a_missing_library_fails_loudly(monkeypatch, tmp_path):
    """Without the built library there is no search at all: loading raises
    instead of falling back to anything on the CPU."""
    monkeypatch.setattr(capi, "_lib", None)
    monkeypatch.setattr(capi, "LIB_PATH", tmp_path / "librivet_me.so")
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        capi.lib()
    with pytest.raises(RuntimeError):
        host.MotionSearch(0)


def test_struct_layouts_match_the_header():
    assert C.sizeof(capi.Mv) == 4
    assert C.sizeof(capi.Result) == 32
    assert C.sizeof(capi.Job) == 28 + 4 * 2 + 4 * capi.RME_MAX_SEEDS
    assert C.sizeof(capi.Params) == 19 * 4


def test_defaults_are_the_oracles():
    for codec, qp in [(capi.RME_CODEC_H264, 28), (capi.RME_CODEC_HEVC, 32)]:
        a, b = capi.default_params(codec, qp), oracle.params(codec, qp)
        for name, _ in capi.Params._fields_:
            assert getattr(a, name) == getattr(b, name), name


@pytest.mark.parametrize("codec,w,h,mask,amp", [(capi.RME_CODEC_HEVC, 1920, 1080, 0xF, 0),
                                                (capi.RME_CODEC_HEVC, 200, 136, 0b1010, 0),
                                                (capi.RME_CODEC_HEVC, 200, 136, 0xF, 0b0101),
                                                (capi.RME_CODEC_HEVC, 136, 200, 0b0111, 0xF),
                                                (capi.RME_CODEC_H264, 352, 288, 0, 0), (capi.RME_CODEC_H264, 100, 70, 0, 0)])
def test_standalone_blocks_are_the_oracles(codec, w, h, mask, amp):
    p = capi.default_params(codec, 30)
    if mask:
        p.hevc_pu_mask = mask
    p.hevc_amp = amp
    got = host.standalone_blocks(codec, w, h, 8, p)
    d = capi.PictureDesc(codec, 8, w, h, w)
    want = oracle.standalone_blocks(d, p)
    np.testing.assert_array_equal(got, want)
    if (codec, w, h, mask) == (capi.RME_CODEC_HEVC, 1920, 1080, 0xF):
        assert len(got) == 32400 + 8040 + 1980 + 480
    if amp:  # two units per enabled mode of every CU of 16 or more, each half of its CU's area
        nmodes = bin(amp).count("1")
        cus = got[got[:, 2] == got[:, 3]]
        big = cus[cus[:, 2] >= 16]
        assert len(got) == len(cus) + 2 * nmodes * len(big)
        units = got[len(cus):]
        assert (units[0::2, 2] * units[0::2, 3] + units[1::2, 2] * units[1::2, 3] ==
                np.repeat(big[:, 2] ** 2, nmodes)).all()


@pytest.mark.parametrize("w,h,mask,nref,amp", [(1920, 1080, 0xF, 2, 0), (200, 136, 0xF, 3, 0), (136, 200, 0b1011, 1, 0),
                                               (200, 136, 0xF, 2, 0b0101)])
def test_the_hevc_decision_is_the_oracles(w, h, mask, nref, amp):
    p = capi.default_params(capi.RME_CODEC_HEVC, 32)
    p.hevc_pu_mask = mask
    p.hevc_amp = amp
    nb = len(host.standalone_blocks(capi.RME_CODEC_HEVC, w, h, 8, p))
    rng = np.random.default_rng(w + h + nref)
    res = np.zeros(nb * nref, capi.RESULT_DTYPE)
    res["cost"] = rng.integers(0, 5000, size=len(res))
    res["cost"][: len(res) // 2 * 2: 2] = res["cost"][1: len(res) // 2 * 2: 2]  # ties between references
    best, part = host.hevc_decide(w, h, 8, p, nref, res)
    d = capi.PictureDesc(capi.RME_CODEC_HEVC, 8, w, h, w)
    obest, opart = oracle.hevc_decide(d, p, nref, res)
    np.testing.assert_array_equal(best, obest)
    np.testing.assert_array_equal(part, opart)
    assert set(np.unique(part)) <= {0, 3, 4, 5, 6}


def test_a_context_without_a_device_fails_cleanly():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a device is present")
    except ImportError:
        pass
    h = C.c_void_p()
    assert capi.lib().rme_ctx_create(C.byref(h), 0) == capi.RME_ECUDA


def test_invalid_arguments_are_refused_without_a_device():
    lib = capi.lib()
    n = C.c_int32()
    bad = capi.PictureDesc(7, 8, 64, 64, 64)
    assert lib.rme_standalone_blocks(C.byref(bad), C.byref(capi.default_params(1, 30)), None, C.byref(n)) == capi.RME_EINVAL
    deep = capi.PictureDesc(1, 16, 64, 64, 64)
    assert lib.rme_standalone_blocks(C.byref(deep), C.byref(capi.default_params(1, 30)), None, C.byref(n)) == capi.RME_EINVAL
    d = capi.PictureDesc(1, 8, 64, 64, 64)
    p = capi.default_params(1, 30)
    p.predictor_mode = capi.RME_PRED_GIVEN
    ps = capi.PlaneSet(16, 224 * 224, 224, 80)
    refs = (capi.PlaneSet * 1)(ps)
    # the search without allocation refuses more jobs than its fixed scratch holds
    assert lib.rme_search_given_noalloc(C.byref(d), C.byref(p), C.byref(ps), refs, 1, C.c_void_p(16), 65537,
                                        C.c_void_p(16), None) == capi.RME_EINVAL
    # and a misaligned plane
    mis = capi.PlaneSet(18, 224 * 224, 224, 80)
    assert lib.rme_search_given_noalloc(C.byref(d), C.byref(p), C.byref(mis), refs, 1, C.c_void_p(16), 4,
                                        C.c_void_p(16), None) == capi.RME_EINVAL


@pytest.mark.parametrize("codec,field,value", [
    (1, "qp", 64), (1, "qp", -13), (1, "hevc_search_range", 1025), (1, "hevc_search_rings", 65),
    (1, "hevc_search_range", -1), (1, "hevc_lambda_scale", float("nan")), (1, "hevc_lambda_scale", -1.0),
    (1, "hevc_lambda_scale", float("inf")), (1, "hevc_pad", 81), (1, "hevc_pad", 7),
    (0, "h264_hpel_iters", 65), (0, "h264_qpel_iters", -1), (0, "h264_range", 513), (0, "h264_pad", 33),
    (0, "h264_vertical_range", -2), (0, "h264_refine_ratio", float("nan")),
])
def test_the_search_without_allocation_holds_parameters_to_the_common_limits(codec, field, value):
    """Every bad parameter is refused (RME_EINVAL) before anything reaches a
    device: a QP whose Lagrangian is not finite, an unbounded walk (range,
    rings, refinement iterations) that would make one launch run for ever."""
    lib = capi.lib()
    d = capi.PictureDesc(codec, 8, 64, 64, 64)
    p = capi.default_params(codec, 30)
    p.predictor_mode = capi.RME_PRED_GIVEN
    setattr(p, field, value)
    pad = 80 if codec == 1 else 32
    cols = 64 + 2 * pad
    ps = capi.PlaneSet(16, cols * cols, cols, pad)
    refs = (capi.PlaneSet * 1)(ps)
    assert lib.rme_search_given_noalloc(C.byref(d), C.byref(p), C.byref(ps), refs, 1, C.c_void_p(16), 4,
                                        C.c_void_p(16), None) == capi.RME_EINVAL


def test_distortion_batches_refuse_host_memory():
    """The batched distortion entry points take device pointers only: host
    arrays (or no device at all) are refused before any launch."""
    a = np.zeros((16, 16), np.uint8)
    off = np.zeros(1, np.int64)
    out = np.zeros(1, np.uint32)
    lib = capi.lib()
    for fn in (lib.rme_sad_batch, lib.rme_satd_batch):
        rc = fn(capi.ptr(a), 16, off.ctypes.data, capi.ptr(a), 16, off.ctypes.data, 8, 8, 8, 1,
                out.ctypes.data_as(C.POINTER(C.c_uint32)), None)
        assert rc == capi.RME_EINVAL
    # satd needs whole 4x4 tiles
    assert lib.rme_satd_batch(None, 16, None, None, 16, None, 6, 8, 8, 0, None, None) == capi.RME_EINVAL
    assert lib.rme_sad_batch(None, 16, None, None, 16, None, 6, 8, 8, 0, None, None) == 0


def test_the_serving_loop_validates_its_arguments():
    lib = capi.lib()
    h = C.c_void_p()
    o = capi.ServeOpts(1 << 30, 8, 4)
    assert lib.rme_serve_start(None, C.byref(o), C.byref(h)) == capi.RME_EINVAL
    bad = capi.ServeOpts(1 << 30, 0, 4)  # no frames per launch
    assert lib.rme_serve_start(C.c_void_p(16), C.byref(bad), C.byref(h)) == capi.RME_EINVAL
    n = C.c_int32()
    assert lib.rme_serve_poll(None, None, 0, C.byref(n)) == capi.RME_EINVAL
    assert lib.rme_serve_submit(None, 1, None, None, None) == capi.RME_EINVAL
    assert lib.rme_serve_stop(None) == capi.RME_EINVAL
