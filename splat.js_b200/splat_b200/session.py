"""Session-level helpers of src/session.js that sit beside the trainer.

``undistort_frames`` mirrors ``undistortFrames(frames, recon)``
(src/session.js:44-80): the same arguments, the same in-place effect on each
frame's ``rgb``, the same return value; the resample runs on the GPU through
``gs_undistort_frames``.  ``cam_position`` is ``camPosition`` (:31-37).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import native as N


def cam_position(pose):
    """World-space position -R^T t of a camera pose {R, t} (session.js:31-37)."""
    R, t = pose["R"], pose["t"]
    return [-(R[0] * t[0] + R[3] * t[1] + R[6] * t[2]),
            -(R[1] * t[0] + R[4] * t[1] + R[7] * t[2]),
            -(R[2] * t[0] + R[5] * t[1] + R[8] * t[2])]


def undistort_frames(frames, recon, device: int = 0) -> bool:
    """Undistort training frames in place (bilinear resample through
    D = 1 + k1 r^2 + k2 r^4) so the pinhole trainer matches the
    reconstruction's distortion-corrected geometry.

    frames: list of dicts {tw, th, fw, rgb (float32, 3*tw*th)}; recon: dict
    {k1, k2, fFeat}.  Returns True when a resample happened (|k1| or |k2| at
    least 0.01); out-of-frame pixels become -1 in every channel, the sentinel
    setup() excludes from the loss.  Each frame's ``rgb`` is replaced by a
    new float32 array, as the reference assigns ``im.rgb = dst``."""
    k1, k2 = float(recon["k1"]), float(recon["k2"])
    if abs(k1) < 0.01 and abs(k2) < 0.01:
        return False
    bufs = [np.array(im["rgb"], dtype=np.float32, copy=True).reshape(-1) for im in frames]
    for im, b in zip(frames, bufs):
        if b.size != 3 * int(im["tw"]) * int(im["th"]):
            raise ValueError("undistort_frames: rgb must hold 3 * tw * th floats")
    arr = (N.GsFrame * max(1, len(frames)))()
    for k, (im, b) in enumerate(zip(frames, bufs)):
        arr[k].tw, arr[k].th, arr[k].fw = int(im["tw"]), int(im["th"]), float(im["fw"])
        arr[k].rgb = b.ctypes.data_as(C.POINTER(C.c_float))
    done = C.c_int32(0)
    N.check(N.lib().gs_undistort_frames(device, arr, len(frames), k1, k2, float(recon["fFeat"]), C.byref(done)))
    for im, b in zip(frames, bufs):
        im["rgb"] = b
    return bool(done.value)
