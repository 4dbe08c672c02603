"""Generate the golden fixtures that freeze the oracle's outputs.

The reference ships no golden motion vectors (its search tests are property
tests), so these fixtures pin the oracle against itself over time: seeded
inputs, the oracle's STANDALONE results and plane samples, written as
compressed npz. Run from the repository root:
    python tests/golden/make_golden.py
and commit the .npz files it writes beside this script.
"""
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path[:0] = [str(ROOT), str(ROOT / "oracle")]

import oracle  # noqa: E402
from rivet_h26x_codecs_b200 import synth  # noqa: E402


def cases():
    """(name, codec, bit_depth, frames, nref, params kwargs)"""
    h = synth.make_sequence(synth.H264, 96, 64, 8, 3, 0x6001, 16, 48, 2.0)
    yield "h264_96x64_medium", synth.H264, 8, h.frames, 2, {}
    yield "h264_96x64_umh", synth.H264, 8, h.frames, 2, {"h264_umh": 1}
    e = synth.make_sequence(synth.HEVC, 128, 96, 8, 3, 0x6002, 64, 96, 2.0)
    yield "hevc_128x96_medium", synth.HEVC, 8, e.frames, 2, {"hevc_search_range": 64}
    yield "hevc_128x96_rings_cross", synth.HEVC, 8, e.frames, 2, {"hevc_search_rings": 1, "hevc_quarter_cross": 1}
    t = synth.make_sequence(synth.HEVC, 96, 64, 10, 3, 0x6003, 64, 96, 6.0)
    yield "hevc_96x64_10bit", synth.HEVC, 10, t.frames, 2, {}


def main():
    for name, codec, bd, frames, nref, kw in cases():
        qp = 28 if codec == synth.H264 else 32
        p = oracle.params(codec, qp, **kw)
        src, refs = frames[nref], [frames[nref - 1 - r] for r in range(nref)]
        res = oracle.frame_search(codec, bd, src, refs, p)
        np.savez_compressed(HERE / f"{name}.npz", src=src, refs=np.stack(refs), results=res.view(np.uint8),
                            codec=codec, bit_depth=bd, qp=qp, params=repr(sorted(kw.items())))
        print(name, len(res))
    pic = frames[0]
    planes, ext = oracle.hevc_planes(pic, 10, force_quarter=True)
    np.savez_compressed(HERE / "hevc_planes_96x64_10bit.npz", pic=pic, planes=planes, ext=ext)


if __name__ == "__main__":
    main()
