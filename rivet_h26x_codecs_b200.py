"""Import shim for the package directory `rivet-h26x-codecs_b200/`.

The directory name carries hyphens, which Python cannot import, so this
module stands in for its `__init__`: it points the package search path at
the directory, after which `import rivet_h26x_codecs_b200.host` (and the
other submodules) resolves there, and re-exports the public host API.
"""
import os as _os

__path__ = [_os.path.join(_os.path.dirname(_os.path.abspath(__file__)), "rivet-h26x-codecs_b200")]

from rivet_h26x_codecs_b200.capi import (  # noqa: E402,F401
    RME_CODEC_H264, RME_CODEC_HEVC, RME_PRED_GIVEN, RME_PRED_STANDALONE, default_params, lib,
)

from rivet_h26x_codecs_b200.host import MotionSearch, Server, distortion_batch, hevc_decide, standalone_blocks  # noqa: E402,F401,E501
