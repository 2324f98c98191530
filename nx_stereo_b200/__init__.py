"""nx_stereo_b200: NxStereo's full-search Stage.Disparity path, with
Stage.Rectification and Stage.SpeckleFilter around it and the stages after
them, as CUDA kernels for B200 (sm_100a) behind a C ABI
(include/nx_stereo_b200.h).

The host side mirrors the reference's interfaces: `stage` the Stage behaviour
and settings checker (lib/nx_stereo/stage.ex), `segment` the Segment
behaviour and CudaSegment, the drop-in for NativeSegment
(lib/nx_stereo/segment.ex, lib/nx_stereo/native_segment.ex).
"""
__version__ = "0.1.0"
