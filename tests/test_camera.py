"""The camera the hq frame's rays start from (`crates/lumenwright/src/scene/camera.rs:86-131`):
Minecraft's yaw and pitch convention, a right-handed basis and `look_at`. The view and projection
matrices there serve the raster path only and are not restated. CPU only.
"""

import numpy as np

from lumenwright_b200.request import Camera


def cam(yaw, pitch):
    return Camera((0.0, 0.0, 0.0), yaw, pitch, 70.0)


def close(a, b):
    return np.linalg.norm(np.asarray(a, np.float64) - np.asarray(b, np.float64)) < 1e-5


def test_minecraft_yaw_convention():  # camera.rs:86-92
    assert close(cam(0.0, 0.0).forward(), [0, 0, 1])
    assert close(cam(90.0, 0.0).forward(), [-1, 0, 0])
    assert close(cam(180.0, 0.0).forward(), [0, 0, -1])
    assert close(cam(0.0, 90.0).forward(), [0, -1, 0])


def test_basis_is_right_handed():  # camera.rs:94-104
    f, r, u = cam(30.0, 20.0).basis()
    assert u[1] > 0.0
    assert close(np.cross(r, u), -f), "the camera looks down -z of its own frame"
    _, r, _ = cam(0.0, 0.0).basis()
    assert close(r, [-1, 0, 0]), "facing south, right is west"


def test_straight_down_takes_right_from_the_yaw():  # camera.rs:26-37
    f, r, u = cam(90.0, 90.0).basis()
    assert close(f, [0, -1, 0])
    assert close(r, [0, 0, -1]) and abs(float(np.linalg.norm(u)) - 1.0) < 1e-6


def test_look_at_roundtrip():  # camera.rs:124-130
    yaw, pitch = Camera.look_at((0.0, 0.0, 0.0), (-5.0, -5.0, 5.0))
    d = np.array([-1.0, -1.0, 1.0]) / np.sqrt(3.0)
    assert close(cam(yaw, pitch).forward(), d)
