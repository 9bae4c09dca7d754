"""Host-side checks of the camera-trace C ABI (no GPU calls): slot counts of the 8x4 tile
order, and argument validation of the camera forward, backward and slot-order entries."""
import ctypes
import math

import numpy as np

from ever_b200 import _native as N
from ever_b200 import camera as CAM


def _cam(w, h, fx=50.0, fy=50.0):
    c = N.EverCamera()
    c.width, c.height, c.fx, c.fy = w, h, fx, fy
    c.cx, c.cy = w / 2, h / 2
    c.c2w = (ctypes.c_float * 12)(1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, -3)
    return c


def test_camera_slot_counts():
    lib = N.load()
    for w, h in ((37, 23), (8, 4), (1, 1), (1920, 1080), (9, 5), (65, 129)):
        want = math.ceil(w / 64) * math.ceil(h / 64) * 4096
        assert lib.ever_camera_slots(ctypes.byref(_cam(w, h))) == want
    assert lib.ever_camera_slots(ctypes.byref(_cam(0, 5))) == 0
    assert lib.ever_camera_slots(ctypes.byref(_cam(4, 4, fx=0.0))) == -1
    assert b"focal" in lib.ever_last_error()
    assert lib.ever_camera_slots(None) == -1
    assert lib.ever_camera_slots(ctypes.byref(_cam(1 << 16, 1 << 15))) == -1  # 2^31 pixels
    assert CAM.camera_slots(CAM.Camera(130, 23, 40.0, 40.0, np.eye(4))) == 3 * 4096


def test_camera_from_view_matches_camera2rays_focal_lengths():
    class V:
        image_width, image_height, FoVx, FoVy = 320, 200, math.radians(60), math.radians(40)
        world_view_transform = np.eye(4)

    c = CAM.Camera.from_view(V)
    assert c.width == 320 and c.height == 200
    assert abs(c.fx - 160 / math.tan(math.radians(30))) < 1e-9
    assert abs(c.fy - 100 / math.tan(math.radians(20))) < 1e-9
    raw = c.c()
    assert raw.cx == 160.0 and raw.cy == 100.0


def test_camera_trace_validation():
    lib = N.load()
    sc = N.EverScene()
    sc.num_prims, sc.sh_coeffs = 0, 1
    args = N.EverTraceArgs()
    args.max_iters, args.sh_degree = 10, -1
    out = N.EverForwardOut()
    cam = _cam(4, 4)
    assert lib.ever_trace_forward_camera(None, ctypes.byref(cam), None, ctypes.byref(args), None,
                                         ctypes.byref(out), None) == 1
    assert lib.ever_trace_forward_camera(ctypes.byref(sc), ctypes.byref(cam), None, ctypes.byref(args), None,
                                         ctypes.byref(out), None) == 1
    assert b"null out" in lib.ever_last_error()
    assert lib.ever_trace_forward_camera(ctypes.byref(sc), None, None, ctypes.byref(args), None,
                                         ctypes.byref(out), None) == 1
    assert b"camera" in lib.ever_last_error()
    # an empty image: nothing to launch
    assert lib.ever_trace_forward_camera(ctypes.byref(sc), ctypes.byref(_cam(0, 4)), None, ctypes.byref(args),
                                         None, ctypes.byref(out), None) == 0
    bout = N.EverBackwardOut()
    rc = lib.ever_trace_backward_camera(ctypes.byref(sc), ctypes.byref(cam), None, ctypes.byref(args), None, None,
                                        None, None, 10, None, 0, None, None, None, None, 0, None, None,
                                        ctypes.byref(bout), None)
    assert rc == 1 and b"ray-side" in lib.ever_last_error()
    # ray gradients: both or neither
    fake = ctypes.c_void_p(256)
    bout.drayo = fake
    rc = lib.ever_trace_backward_camera(ctypes.byref(sc), ctypes.byref(cam), None, ctypes.byref(args), fake, fake,
                                        fake, fake, 10, None, 0, None, None, None, None, 0, None, None,
                                        ctypes.byref(bout), None)
    assert rc == 1 and b"ray-side" in lib.ever_last_error()
    ws_need = lib.ever_ray_order_workspace_bytes(lib.ever_camera_slots(ctypes.byref(cam)))
    assert lib.ever_camera_backward_slot_order(ctypes.byref(cam), fake, 0, fake, ws_need - 1, fake, None) == 3
    assert lib.ever_camera_backward_slot_order(ctypes.byref(cam), fake, 17, fake, ws_need, fake, None) == 1
    assert lib.ever_camera_slot_pixels(ctypes.byref(cam), None, None) == 1
    assert lib.ever_camera_event_log_to_reference(None, ctypes.byref(cam), None, 0, None, None, 5, None) == 1


def test_camera_regrouped_validation():
    lib = N.load()
    sc = N.EverScene()
    sc.num_prims, sc.sh_coeffs = 0, 1
    args = N.EverTraceArgs()
    args.max_iters, args.sh_degree = 10, -1
    out = N.EverForwardOut()
    fake = ctypes.c_void_p(256)
    out.out, out.iters = fake, fake
    cam = _cam(4, 4)
    rc = lib.ever_trace_forward_camera_regrouped(ctypes.byref(sc), ctypes.byref(cam), None, ctypes.byref(args), None,
                                                 ctypes.byref(out), None, 0, None)
    assert rc == 1 and b"states" in lib.ever_last_error()
    out.states, out.last_dirac = fake, fake
    need = lib.ever_trace_forward_workspace_bytes(lib.ever_camera_slots(ctypes.byref(cam)))
    rc = lib.ever_trace_forward_camera_regrouped(ctypes.byref(sc), ctypes.byref(cam), None, ctypes.byref(args), None,
                                                 ctypes.byref(out), fake, need - 1, None)
    assert rc == 3
    rc = lib.ever_trace_forward_regrouped(ctypes.byref(sc), fake, fake, 100, ctypes.byref(args), None, None,
                                          ctypes.byref(out), fake, 0, None)
    assert rc == 3 and b"workspace" in lib.ever_last_error()
    assert lib.ever_trace_forward_workspace_bytes(-1) == 0 and lib.ever_trace_forward_workspace_bytes(1 << 31) == 0
